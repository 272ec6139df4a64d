"""Parity of the sm_100a tile-staged elastic Newmark path against the CPU oracle.

Tolerances (relative L2):
* seismograms and the displacement field: 1e-5 against the FP32 oracle (the
  FP32 restatement of the reference CPU solver) and against the reference's
  own REF_SEIS traces;
* velocity and acceleration fields late in a run: two FP32 builds that differ
  only in rounding (for instance FMA contraction on or off) drift apart by
  up to ~6e-5 (velocity) and ~8e-4 (acceleration) after 3000 steps, as much as
  FP32 drifts from FP64.  These fields must be as accurate as the FP32 oracle:
  their error against the FP64 oracle may exceed the FP32 oracle's own error
  against FP64 by at most 50 %.
"""
import numpy as np
import pytest

from helpers import load_golden, rel_l2
from specfem2d_b200.setup.from_par_file import database_from_config

pytestmark = pytest.mark.gpu
TOL = 1e-5


@pytest.fixture(scope="module")
def tromp():
    cfg, seis = load_golden("tromp2005_kernel")
    return database_from_config(cfg), seis


@pytest.fixture(scope="module")
def tromp_oracle(tromp):
    import oracle

    db, _ = tromp
    o = oracle.Oracle(db, 4)
    s = o.run(db.nstep)
    o64 = oracle.Oracle(db, 8)
    o64.run(db.nstep)
    return s, o.displ.copy(), o.veloc.copy(), o.accel.copy(), o64.veloc.copy(), o64.accel.copy()


def test_tromp_seismograms_match_oracle_and_golden(tromp, tromp_oracle):
    from specfem2d_b200.runtime import ElasticSolver

    db, golden = tromp
    s_or = tromp_oracle[0]
    sol = ElasticSolver(db)
    s = sol.run(db.nstep)
    for c in range(2):
        assert rel_l2(s[0, :, c], s_or[0, :, c]) < TOL
    assert rel_l2(s[0, :, 0], golden["S0001_BXX"]) < TOL
    assert rel_l2(s[0, :, 1], golden["S0001_BXZ"]) < TOL
    d, v, a = sol.get_fields()
    assert rel_l2(d, tromp_oracle[1]) < TOL
    v64, a64 = tromp_oracle[4], tromp_oracle[5]
    assert rel_l2(v, v64) < 1.5 * rel_l2(tromp_oracle[2], v64)
    assert rel_l2(a, a64) < 1.5 * rel_l2(tromp_oracle[3], a64)


@pytest.fixture(scope="module")
def oracle_1500(tromp):
    import oracle

    db, _ = tromp
    # the P wave reaches the receiver (100 km away) after about 1250 steps
    o = oracle.Oracle(db, 4)
    ref = o.run(1500)
    o64 = oracle.Oracle(db, 8)
    o64.run(1500)
    return ref, o.displ.copy(), o.veloc.copy(), o64.veloc.copy()


@pytest.mark.parametrize("tile_elems,threads", [(8, 128), (25, 256), (64, 512), (128, 256), (32, 250), (10, 250)])
def test_tile_size_invariance(tromp, oracle_1500, tile_elems, threads):
    from specfem2d_b200.runtime import ElasticSolver

    db, _ = tromp
    ref, d_or, v_or, v64 = oracle_1500
    sol = ElasticSolver(db, tile_elems=tile_elems, threads_per_block=threads)
    s = sol.run(1500)
    assert rel_l2(s, ref) < TOL
    d, v, _ = sol.get_fields()
    assert rel_l2(d, d_or) < TOL
    assert rel_l2(v, v64) < 1.5 * rel_l2(v_or, v64)


def test_bitwise_deterministic_and_chunking(tromp):
    from specfem2d_b200.runtime import ElasticSolver

    db, _ = tromp
    a = ElasticSolver(db).run(500)
    sol = ElasticSolver(db)
    b1 = sol.run(123)
    b2 = sol.run(377)
    b = np.concatenate([b1, b2], axis=1)
    assert np.array_equal(a, b)


def test_set_get_fields_roundtrip_and_restart(tromp):
    import oracle
    from specfem2d_b200.runtime import ElasticSolver

    db, _ = tromp
    rng = np.random.default_rng(0)
    d0 = (rng.standard_normal((db.nglob, 2)) * 1e-6).astype(np.float32)
    sol = ElasticSolver(db)
    sol.set_fields(d0, None, None)
    d, v, a = sol.get_fields()
    assert np.array_equal(d, d0) and not v.any() and not a.any()
    # restart from a random displacement: compare with the oracle
    o = oracle.Oracle(db, 4)
    o.set(oracle.DISPL, d0)
    ref = o.run(100)
    s = sol.run(100)
    assert rel_l2(s, ref) < TOL
    d, _, _ = sol.get_fields()
    assert rel_l2(d, o.displ) < TOL


def test_unstable_is_reported(tromp):
    from specfem2d_b200.runtime import ElasticSolver, UnstableError

    db, _ = tromp
    sol = ElasticSolver(db)
    bad = np.zeros((db.nglob, 2), dtype=np.float32)
    bad[db.nglob // 2] = np.nan
    sol.set_fields(bad, None, None)
    with pytest.raises(UnstableError):
        sol.run(3)


def test_solvers_with_different_tile_sizes_coexist(tromp):
    """The tile kernel's shared-memory limit is per kernel, not per solver: a
    solver with small tiles created after one with large tiles must not break
    the launches of the first."""
    from specfem2d_b200.runtime import ElasticSolver

    db, _ = tromp
    big = ElasticSolver(db, tile_elems=128)
    small = ElasticSolver(db, tile_elems=8)
    a = big.run(64)
    b = small.run(64)
    assert rel_l2(a, b) < TOL
    big.close()
    small.close()


def test_initialize_device_selects_rank_modulo_devices(tromp):
    """sf2d_initialize_device (initialize_cuda_device): rank % visible devices
    becomes current in the library's runtime, and a solver created afterwards
    runs on it; a negative rank is an error."""
    import torch

    from specfem2d_b200.runtime import ElasticSolver, SF2DError, initialize_device

    n = initialize_device(0)
    assert n == torch.cuda.device_count() and n >= 1
    assert initialize_device(n) == n  # rank n wraps to device 0
    db, _ = tromp
    s = ElasticSolver(db)
    assert np.isfinite(s.run(10)).all()
    with pytest.raises(SF2DError):
        initialize_device(-1)
