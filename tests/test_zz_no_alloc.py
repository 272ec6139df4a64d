"""sf2d_member_norms_noalloc against the solver's own sf2d_get_norm.

The entry point serves callers that cannot let a library allocate device
memory mid-run (their device memory is planned up front or held by a pooling
allocator), so it keeps its intermediates in a static device array.  This
file is collected last on purpose: the entry point looks that array up on its
first call on a device, so it must work both in a fresh process (run this file
alone) and after every other test has created and destroyed solvers.
"""
import numpy as np
import pytest

from specfem2d_b200 import batch
from specfem2d_b200.configs import random_layered_model

# three independent layered models of different sizes, one batch
SIZES = [(11, 60, 30), (12, 40, 24), (13, 50, 20)]
NSTEP = 600


def _members():
    return [random_layered_model(seed, nx, nz, NSTEP) for seed, nx, nz in SIZES]


@pytest.mark.gpu
def test_member_norms_match_get_norm_on_two_calls():
    import torch

    from specfem2d_b200.runtime import ElasticSolver, member_norms_noalloc

    members = _members()
    packed, idx = batch.pack(members)
    whole = ElasticSolver(packed)
    singles = [ElasticSolver(m) for m in members]
    free = []
    for call, nrun in enumerate((300, 300)):
        whole.run(nrun, seismograms=False)
        for s in singles:
            s.run(nrun, seismograms=False)
        displ, _, _ = whole.get_fields()
        field = torch.from_numpy(np.ascontiguousarray(displ, dtype=np.float32)).cuda()
        torch.cuda.synchronize()
        free.append(torch.cuda.mem_get_info()[0])
        stream = 0 if call == 0 else whole.stream_handle()
        got = member_norms_noalloc(field.data_ptr(), idx.glob_off, stream=stream)
        free.append(torch.cuda.mem_get_info()[0])
        # the batch-wide maximum equals the batched solver's own norm
        assert float(got.max()) == pytest.approx(whole.max_norm(), rel=1e-6)
        # each member's maximum matches that member run alone (FP32 noise only)
        for m, s in enumerate(singles):
            ref = s.max_norm()
            assert ref > 0.0
            assert abs(float(got[m]) - ref) <= 1e-4 * ref, (call, m, float(got[m]), ref)
    # the second call leaves the device's free memory unchanged
    assert free[2] == free[3]
    whole.close()
    for s in singles:
        s.close()


@pytest.mark.gpu
def test_member_norms_edge_cases_and_rejections():
    import torch

    from specfem2d_b200.runtime import SF2DError, member_norms_noalloc

    n = 1000
    u = torch.zeros((n, 2), dtype=torch.float32, device="cuda")
    u[10] = torch.tensor([3.0, 4.0])             # member 0: norm 5
    u[700] = torch.tensor([float("nan"), 0.0])   # member 2: NaN counts as +inf
    torch.cuda.synchronize()
    # an empty member in the middle and a range that starts past point 0
    got = member_norms_noalloc(u.data_ptr(), [5, 600, 600, n])
    assert got[0] == 5.0 and got[1] == 0.0 and np.isinf(got[2])
    # one member
    assert member_norms_noalloc(u.data_ptr(), [0, 600])[0] == 5.0
    # beyond the static scratch, decreasing offsets, no member, beyond the allocation
    big = np.zeros(4097 + 1, dtype=np.int64)
    # the last offset near INT64_MAX / 8 wraps 8 * offset past 2^64: it must still be rejected
    for bad in (big, [0, 10, 5], [0], [0, 1 << 40], [0, (1 << 63) // 8 - 1], [0, (1 << 63) - 1]):
        with pytest.raises(SF2DError):
            member_norms_noalloc(u.data_ptr(), bad)
