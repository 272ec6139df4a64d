"""Kernel smoothing (smooth_sem.F90:63-467): the oracle's restatement of the
reference's CPU loop (every pair of points, CUSTOM_REAL) and the GPU kernel
(sf2d_smooth: cells of `cutoff` standard deviations, double sums).

No reference output pins the smoothing (the reference ships no smoothed
kernel files); the oracle follows the CPU program's arithmetic and the GPU is
held to it.  Tolerance: 1e-5 relative L2 (the GPU leaves out weights below
exp(-18) and sums in double; the oracle sums in float)."""
import numpy as np
import pytest

from fwi_case import Case
from helpers import rel_l2


@pytest.fixture(scope="module")
def fields():
    c = Case(nstep=10)
    db = c.start_db()
    rng = np.random.default_rng(0)
    f = np.stack([np.ones((db.nspec, 5, 5)), c.anomaly(), rng.standard_normal((db.nspec, 5, 5)),
                  c.anomaly(2100.0, 1100.0, 150.0) * rng.uniform(0.5, 1.5, (db.nspec, 5, 5))])
    return db, f.astype(np.float32)


def test_oracle_smoothing_keeps_constants_and_averages(fields):
    import oracle

    db, f = fields
    out = oracle.smooth(db, f, 200.0, 100.0)
    assert np.abs(out[0] - 1.0).max() < 1e-6            # a normalised average of a constant
    assert out[1].max() < f[1].max() and out[1].min() >= f[1].min()
    assert out[2].std() < 0.1 * f[2].std()              # white noise averages out
    # every copy of a global point gets the value of the point
    g = db.ibool.ravel()
    v = out[1].ravel()
    first = np.full(db.nglob, -1)
    first[g[::-1]] = np.arange(g.size - 1, -1, -1)
    assert np.array_equal(v, v[first[g]])


@pytest.mark.gpu
@pytest.mark.parametrize("sigmas", [(200.0, 100.0), (150.0, 300.0)])
def test_gpu_smoothing_matches_oracle(fields, sigmas):
    import oracle

    from specfem2d_b200.runtime import smooth

    db, f = fields
    ref = oracle.smooth(db, f, *sigmas)
    got = smooth(db, f, *sigmas)
    for k in range(f.shape[0]):
        assert rel_l2(got[k], ref[k]) < 1e-5, k
