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


def test_pack_rejects_fluid_or_cpml_members():
    """A packed mesh concatenates the solid arrays only: members with fluid
    elements or CPML layers are refused instead of being modelled wrong."""
    cfg, _ = load_golden("pressure_source_acoustic")
    db = database_from_config(cfg)
    assert db.acoustic is not None and db.pml is not None
    with pytest.raises(ValueError):
        batch.pack([db, db])


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


@pytest.mark.gpu
def test_a_failed_member_is_masked_and_the_others_run_on():
    """Failure injected on the host: after 200 steps one member's displacement is
    set to NaN.  With members declared, that member is masked (status 1), the run
    does not fail, and the other members' traces are bit-identical to a run
    without the fault.  Without members the same fault fails the whole run, as
    the reference's check_stability does (check_stability.F90:95-98)."""
    from specfem2d_b200.runtime import ElasticSolver, UnstableError

    c, db, shots = _members()
    packed, idx = batch.pack(shots)
    members = batch.element_members(idx)
    go, ro = idx.glob_off, idx.rec_off

    def run(declare, inject):
        sol = ElasticSolver(packed)
        if declare:
            sol.set_members(members)
        s1 = sol.run(200)
        if inject:
            u, v, a = sol.get_fields()
            u[go[1]:go[2]] = np.nan
            sol.set_fields(u, v, a)
        s2 = sol.run(packed.nstep - 200)
        st = sol.member_status() if declare else None
        sol.close()
        return np.concatenate([s1, s2], axis=1), st

    ref, st0 = run(True, False)
    assert list(st0) == [0, 0, 0]
    got, st = run(True, True)
    assert list(st) == [0, 1, 0]
    for m in (0, 2):
        assert np.array_equal(got[ro[m]:ro[m + 1]], ref[ro[m]:ro[m + 1]])
    with pytest.raises(UnstableError):
        run(False, True)


@pytest.mark.gpu
def test_synchronize_gives_up_with_a_timeout_status():
    """A wait shorter than the queued work returns SF2D_ERR_TIMEOUT; the steps
    keep running and a later wait without a limit finishes them."""
    from specfem2d_b200.runtime import ElasticSolver, SolverTimeout

    c, db, shots = _members()
    sol = ElasticSolver(db)
    sol.enqueue(db.nstep)
    with pytest.raises(SolverTimeout):
        sol.synchronize(1e-5)
    sol.synchronize(0.0)
    assert sol.step_index() == db.nstep
    sol.close()


@pytest.mark.gpu
def test_summed_shot_gradient_matches_the_oracle_sum():
    """The survey gradient of summed_shot_gradient (kernels summed over the shots
    of one model, one packed batch on the GPU) against the sum of the oracle's
    per-shot gradients: as close to the FP64 sum as the FP32 oracle's sum is
    (this case's residual is 0.14 % of the synthetics, so FP32 rounding of the
    synthetics sets the agreement; see test_gradient_gpu)."""
    import oracle

    from specfem2d_b200.fwi import summed_shot_gradient

    c, db, shots = _members()
    truth = batch.shots_on_model(c.true_db(), [(1000.0, 1800.0), (2000.0, 1500.0), (3000.0, 1900.0)], 30.0)
    observed = [oracle.Oracle(t, 8).run(t.nstep) for t in truth]
    chi, rk, kk, mk = summed_shot_gradient(shots, observed, checkpoint_every=100)
    ref64 = [oracle.gradient(s, o, checkpoint_every=100, precision=8) for s, o in zip(shots, observed)]
    ref32 = [oracle.gradient(s, o, checkpoint_every=100, precision=4) for s, o in zip(shots, observed)]
    assert chi == pytest.approx(sum(r[0] for r in ref32), rel=1e-4)
    for k, got in ((2, rk), (3, kk), (4, mk)):
        s64 = sum(r[k].astype(np.float64) for r in ref64)
        s32 = sum(r[k].astype(np.float64) for r in ref32)
        assert rel_l2(got, s64) < 1.5 * rel_l2(s32, s64)


@pytest.mark.gpu
def test_native_batch_forward_matches_the_packed_database():
    """The batch C ABI (sf2d_batch_*): three shots on one model, packed by the
    library, give the traces of the same shots packed on the host (the same
    tiles, so the same arithmetic), and each member matches its own FP32
    oracle run."""
    import oracle
    from specfem2d_b200.runtime import ElasticSolver

    c, db, shots = _members()
    nb = batch.NativeBatch([db], shots=shots, shot_models=[0, 0, 0])
    assert (nb.nmembers, nb.nspec, nb.nglob) == (3, 3 * db.nspec, 3 * db.nglob)
    got = nb.forward()
    again = nb.forward()
    assert np.array_equal(got, again) and list(nb.member_status()) == [0, 0, 0]
    nb.close()
    packed, idx = batch.pack(shots)
    ref = ElasticSolver(packed).run(db.nstep)
    assert rel_l2(got, ref) < 1e-6
    for m, s in enumerate(shots):
        assert rel_l2(got[idx.rec_off[m]:idx.rec_off[m + 1]], oracle.Oracle(s, 4).run(db.nstep)) < 1e-5


@pytest.mark.gpu
def test_native_gradient_batch_sums_the_shots_of_each_model():
    """A gradient batch of two models with shots on each: the kernels come back
    per model, summed over its shots, equal to the per-shot gradients of the
    host-packed batch summed on the host."""
    from specfem2d_b200.fwi import l2_misfit_gradient

    c, db, shots = _members()
    true_db = c.true_db()
    pos = [(1000.0, 1800.0), (2000.0, 1500.0), (3000.0, 1900.0)]
    shots_b = batch.shots_on_model(true_db, pos[:2], angle_deg=30.0)
    members = shots + shots_b
    nb = batch.NativeBatch([db, true_db], shots=members, shot_models=[0, 0, 0, 1, 1], checkpoint_every=100)
    syn = nb.forward()
    obs = 0.9 * syn
    per_model = nb.adjoint(syn - obs)
    nb.close()
    packed, idx = batch.pack(members)
    _, syn_ref, rk, kk, mk = l2_misfit_gradient(packed, obs, checkpoint_every=100)
    assert rel_l2(syn, syn_ref) < 1e-6
    for model, mem in ((0, [0, 1, 2]), (1, [3, 4])):
        for k, arr in enumerate((rk, kk, mk)):
            parts = batch.split_elements(arr, idx)
            ref = sum(parts[m].astype(np.float64) for m in mem)
            assert rel_l2(per_model[model][k], ref) < 1e-5, (model, k)


def test_native_batch_rejects_mismatched_models_before_any_gpu_work():
    """sf2d_batch_create checks its models and shots on the host and returns
    SF2D_ERR_INVALID (no GPU is touched)."""
    c, db, shots = _members()
    other = Case(nstep=400).start_db()
    with pytest.raises(Exception, match="share nstep"):
        batch.NativeBatch([db, other])
    with pytest.raises(Exception, match="shot model out of range"):
        batch.NativeBatch([db], shots=shots[:1], shot_models=[3])
    cfg, _ = load_golden("pressure_source_acoustic")
    with pytest.raises(Exception, match="CPML"):
        fl = database_from_config(cfg)
        fl.acoustic = None  # the CPML check comes first
        batch.NativeBatch([fl])


@pytest.mark.gpu
def test_native_batch_lddrk_members_match_single_runs():
    """An LDDRK batch through the C ABI (6 stages: the packed source time
    functions carry every stage): two models, one of them with its stf scaled,
    give each member the traces of its own run (within the 1e-5 of the FP32 policy)."""
    from specfem2d_b200.runtime import ElasticSolver

    cfg, _ = load_golden("tromp2005_kernel")
    a = database_from_config(cfg, nstep=1500, time_scheme=2)
    b = database_from_config(cfg, nstep=1500, time_scheme=2)
    b.stf = (2.0 * b.stf).astype(b.stf.dtype)
    nb = batch.NativeBatch([a, b])
    got = nb.forward()
    nb.close()
    assert got.shape[0] == len(a.rec_ispec) + len(b.rec_ispec)
    for m, db in enumerate((a, b)):
        ref = ElasticSolver(db).run(db.nstep)
        assert np.abs(ref).max() > 1e-12  # the wave has reached the receiver
        n0 = m * len(a.rec_ispec)
        # a single run tiles the model on its own, so shared points sum in another
        # order: FP32 rounding, 2e-6 after 1500 LDDRK steps
        assert rel_l2(got[n0:n0 + len(db.rec_ispec)], ref) < 1e-5
