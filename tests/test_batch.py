"""Batches packed into one disconnected mesh: host-side checks (CPU) and GPU
parity of batched forward runs and gradients with per-member runs."""
import numpy as np
import pytest

from fwi_case import Case
from helpers import load_golden, rel_l2
from specfem2d_b200 import batch
from specfem2d_b200.setup.from_par_file import database_from_config


def _members():
    c = Case(nstep=500)
    db = c.start_db()
    shots = batch.shots_on_model(db, [(1000.0, 1800.0), (2000.0, 1500.0), (3000.0, 1900.0)], angle_deg=30.0)
    return c, db, shots


def test_pack_offsets_and_tiling():
    from specfem2d_b200.runtime import tiling_stats

    c, db, shots = _members()
    packed, idx = batch.pack(shots)
    assert packed.nspec == 3 * db.nspec and packed.nglob == 3 * db.nglob
    assert packed.ibool.max() == packed.nglob - 1
    assert list(idx.rec_off) == [0, 9, 18, 27]
    st = tiling_stats(packed, 32)
    assert st["n_interior"] + st["nshared"] == packed.nglob
    # each member keeps its own source
    assert list(packed.source_ispec - idx.elem_off[:3]) == [s.source_ispec[0] for s in shots]


def test_pack_rejects_mismatched_members():
    c, db, shots = _members()
    other = Case(nstep=400).start_db()
    with pytest.raises(ValueError):
        batch.pack([shots[0], other])


@pytest.mark.gpu
def test_batched_forward_matches_members():
    import oracle
    from specfem2d_b200.runtime import ElasticSolver

    c, db, shots = _members()
    packed, idx = batch.pack(shots)
    got = batch.split_seismograms(ElasticSolver(packed).run(db.nstep), idx)
    for m, s in enumerate(shots):
        ref = oracle.Oracle(s, 4).run(db.nstep)
        assert rel_l2(got[m], ref) < 1e-5


@pytest.mark.gpu
def test_batched_gradient_matches_members():
    import oracle
    from specfem2d_b200.fwi import l2_misfit_gradient

    c, db, shots = _members()
    true_shots = batch.shots_on_model(c.true_db(), [(1000.0, 1800.0), (2000.0, 1500.0), (3000.0, 1900.0)],
                                      angle_deg=30.0)
    obs = [oracle.Oracle(t, 8).run(c.nstep) for t in true_shots]
    packed, idx = batch.pack(shots)
    chi, seis, rk, kk, mk = l2_misfit_gradient(packed, np.concatenate(obs, axis=0), checkpoint_every=100)
    # summed gradient over the shots versus per-shot FP64 oracle gradients
    ref64 = [oracle.gradient(s, o, checkpoint_every=100, precision=8) for s, o in zip(shots, obs)]
    ref32 = [oracle.gradient(s, o, checkpoint_every=100, precision=4) for s, o in zip(shots, obs)]
    for k, got in ((2, rk), (3, kk), (4, mk)):
        parts = batch.split_elements(got, idx)
        gsum = sum(p.astype(np.float64) for p in parts)
        s64 = sum(r[k].astype(np.float64) for r in ref64)
        s32 = sum(r[k].astype(np.float64) for r in ref32)
        assert rel_l2(gsum, s64) < 1.5 * rel_l2(s32, s64)
    assert abs(chi - sum(r[0] for r in ref32)) / chi < 1e-4
