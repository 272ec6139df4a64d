"""Parity of the coupled fluid-solid GPU path (fluid tile solver + solid tile
solver + coupling edges) against the CPU oracle and the reference's own traces.

Tolerance policy (relative L2), as for the solid path: FP32 runs that differ
only in rounding drift apart by about as much as FP32 drifts from FP64, so
each GPU result must be at most 1.5-2x as far from the FP64 oracle as the
FP32 oracle is, or within 1e-5 of the FP32 oracle.
"""
import os

import numpy as np
import pytest

from helpers import load_golden, rel_l2
from specfem2d_b200 import configs
from specfem2d_b200.setup.from_par_file import database_from_config

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def _ocean():
    cfg, seis = load_golden("tomographic_ocean_model")
    t = np.load(os.path.join(HERE, "golden", "tomographic_ocean_model_tomo.npz"))
    db = database_from_config(cfg, tomo=(t["x"], t["z"], t["vp"], t["vs"], t["rho"]))
    return db, seis


def test_ocean_model_matches_oracle_and_ref_seis():
    """EXAMPLES/tomographic_ocean_model: displacement receivers in the water
    (from grad chi / rho) and in the rock, 1600 steps."""
    import oracle
    from specfem2d_b200.coupled import CoupledSolver

    db, seis = _ocean()
    gpu = CoupledSolver(db).run(db.nstep)
    o32 = oracle.Oracle(db, 4).run(db.nstep)
    o64 = oracle.Oracle(db, 8).run(db.nstep)
    assert rel_l2(gpu, o64) < 2.0 * rel_l2(o32, o64)
    stations = (1, 3, 6, 9, 12, 14, 16, 18, 20, 22)
    g, r = [], []
    for k in stations:
        for c, ci in (("BXX", 0), ("BXZ", 1)):
            g.append(gpu[k - 1, :, ci])
            r.append(seis[f"S{k:04d}_{c}"])
    assert rel_l2(np.concatenate(g), np.concatenate(r)) < 3e-5


@pytest.fixture(scope="module")
def c2_small():
    return configs.c2_coupled(nstep=1500, nrec=24, scale=8)


def _close(gpu, ref, ref64):
    return rel_l2(gpu, ref) < 1e-5 or rel_l2(gpu, ref64) < 1.5 * rel_l2(ref, ref64)


def test_pressure_traces_and_fields_match_oracle(c2_small):
    """Pressure source in the water, pressure receivers: traces and fields as
    accurate as the FP32 oracle."""
    import oracle
    from specfem2d_b200.coupled import CoupledSolver

    db = c2_small
    s = CoupledSolver(db)
    gpu = s.run(db.nstep)
    f = s.get_fields()
    o32 = oracle.Oracle(db, 4)
    ref = o32.run(db.nstep)
    o64 = oracle.Oracle(db, 8)
    ref64 = o64.run(db.nstep)
    assert np.abs(ref).max() > 0 and np.all(gpu[:, :, 1] == 0.0)
    assert _close(gpu, ref, ref64)
    for name, which in (("pot", oracle.POT), ("pot_dot", oracle.POT_DOT)):
        a64 = o64.get(which)
        assert rel_l2(f[name], a64) < 1.5 * rel_l2(o32.get(which), a64) + 1e-7, name
    assert rel_l2(f["displ"], o64.displ) < 1.5 * rel_l2(o32.displ, o64.displ) + 1e-7


def test_use_trick_pressure():
    """USE_TRICK_FOR_BETTER_PRESSURE: d2-Ricker source, pressure = -chi."""
    import oracle
    from specfem2d_b200.coupled import CoupledSolver

    db = configs.c2_coupled(nstep=800, nrec=12, scale=8, use_trick=True)
    gpu = CoupledSolver(db).run(db.nstep)
    ref = oracle.Oracle(db, 4).run(db.nstep)
    ref64 = oracle.Oracle(db, 8).run(db.nstep)
    assert _close(gpu, ref, ref64)


def test_lddrk_coupled_matches_oracle():
    import oracle
    from specfem2d_b200.coupled import CoupledSolver

    db = configs.c2_coupled(nstep=600, nrec=12, scale=8, time_scheme=2)
    gpu = CoupledSolver(db).run(db.nstep)
    ref = oracle.Oracle(db, 4).run(db.nstep)
    ref64 = oracle.Oracle(db, 8).run(db.nstep)
    assert _close(gpu, ref, ref64)


def test_restart_and_chunking_bitwise(c2_small):
    """Running 200 steps in pieces (graph chunks plus remainders) gives the
    same bits as one call; fields round-trip through get/set."""
    from specfem2d_b200.coupled import CoupledSolver

    db = c2_small
    a = CoupledSolver(db).run(200)
    s = CoupledSolver(db)
    b = np.concatenate([s.run(37), s.run(100), s.run(63)], axis=1)
    assert np.array_equal(a, b)
    f = s.get_fields()
    s2 = CoupledSolver(db)
    s2.set_fields(**f)
    g = s2.get_fields()
    for k in f:
        assert np.array_equal(f[k], g[k]), k
