"""The reference's own Fortran-to-GPU interface (include/sf2d_fortran.h), driven
the way the SPECFEM2D Fortran host drives it (tests/fortran_driver.py: the
call order of prepare_gpu.f90, iterate_time.F90, compute_gpu_elastic.f90 and
write_seismograms.F90, arguments by reference, 1-based indices, Fortran array
order).  No Fortran compiler is needed: the calls are the C symbols gfortran
would make.

Tolerances (relative L2): the reference's REF_SEIS traces within 1e-5; the
same run through this library's own C ABI within 1e-5 (the interface forms
lambda = kappa - mu in FP32 as the reference's GPU kernel does, the C ABI
takes lambda as the CPU solver forms it).
"""
import numpy as np
import pytest

from fortran_driver import run_forward
from helpers import load_golden, rel_l2
from specfem2d_b200.setup.from_par_file import database_from_config

pytestmark = pytest.mark.gpu


def test_tromp2005_through_the_fortran_interface_matches_ref_seis():
    from specfem2d_b200.runtime import ElasticSolver

    cfg, golden = load_golden("tromp2005_kernel")
    db = database_from_config(cfg)
    seis, displ, norms = run_forward(db)
    assert rel_l2(seis[0, :, 0], golden["S0001_BXX"]) < 1e-5
    assert rel_l2(seis[0, :, 1], golden["S0001_BXZ"]) < 1e-5
    sol = ElasticSolver(db)
    s = sol.run(db.nstep)
    d, _, _ = sol.get_fields()
    assert rel_l2(seis, s) < 1e-5
    assert rel_l2(displ, d) < 1e-5
    assert len(norms) == 3 and norms[-1] > 0


def test_seismogram_buffer_flushes_match_one_buffer():
    """NTSTEP_BETWEEN_OUTPUT_SEISMOS shorter than the run: the host's trace
    buffer is handed over five times; the traces are those of one buffer."""
    cfg, _ = load_golden("tromp2005_kernel")
    db = database_from_config(cfg, nstep=1400)
    a, _, _ = run_forward(db)
    b, _, _ = run_forward(db, nlength_seismogram=300)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("name", ["anisotropic_isotropic_model", "attenuation_viscoelastic"])
def test_anisotropic_and_attenuating_examples_through_the_fortran_interface(name):
    """Anisotropic elements (c_ij arrays of prepare_fields_elastic_device) and
    3-SLS attenuation (its A/B Newmark arrays), against the FP32 oracle."""
    import oracle

    cfg, _ = load_golden(name)
    db = database_from_config(cfg, absorbing_as_stacey=True)
    seis, displ, _ = run_forward(db)
    o = oracle.Oracle(db, 4)
    ref = o.run(db.nstep)
    assert rel_l2(seis, ref) < 1e-5
    assert rel_l2(displ, o.displ) < 1e-5


def _ocean_db():
    import os

    cfg, seis = load_golden("tomographic_ocean_model")
    t = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "tomographic_ocean_model_tomo.npz"))
    return database_from_config(cfg, tomo=(t["x"], t["z"], t["vp"], t["vs"], t["rho"])), seis


def test_coupled_ocean_through_the_fortran_interface():
    """EXAMPLES/tomographic_ocean_model (fluid over rock: coupling both ways,
    Stacey in both domains, a free sea surface, displacement receivers in both)
    through prepare_fields_acoustic_device and compute_gpu_acoustic.f90's call
    order: within the FP32 band of the FP64 oracle, and the reference's traces
    as close as the coupled GPU solver gets them."""
    import oracle

    db, seis = _ocean_db()
    out, displ, norms, pot = run_forward(db, check_every=400)
    o32 = oracle.Oracle(db, 4)
    ref32 = o32.run(db.nstep)
    ref64 = oracle.Oracle(db, 8).run(db.nstep)
    assert rel_l2(out, ref64) < 2.0 * rel_l2(ref32, ref64)
    g, r = [], []
    for k in (1, 3, 6, 9, 12, 14, 16, 18, 20, 22):
        for c, ci in (("BXX", 0), ("BXZ", 1)):
            g.append(out[k - 1, :, ci])
            r.append(seis[f"S{k:04d}_{c}"])
    assert rel_l2(np.concatenate(g), np.concatenate(r)) < 3e-5
    assert rel_l2(pot, o32.get(oracle.POT)) < 1e-4
    assert len(norms) == 4 and all(a > 0 and b > 0 for a, b in norms)


def test_fluid_only_external_mesh_through_the_fortran_interface():
    """EXAMPLES/Gmsh_example_Stacey_MPI (fluid only: the fused step is queued by
    kernel_3_acoustic_cuda), pressure receivers, the listed free surface."""
    import oracle

    cfg, seis = load_golden("gmsh_stacey_external")
    db = database_from_config(cfg)
    out, _, norms, pot = run_forward(db, check_every=600)
    o32 = oracle.Oracle(db, 4).run(db.nstep)
    o64 = oracle.Oracle(db, 8).run(db.nstep)
    for k in range(11):
        band = rel_l2(o32[k, :, 0], o64[k, :, 0])
        assert rel_l2(out[k, :, 0], o64[k, :, 0]) < 1.5 * band
        assert rel_l2(out[k, :, 0], seis[f"S{k + 1:04d}_PRE"]) < 2.0 * band
    assert np.all(out[:, :, 1] == 0.0) and norms[-1][0] == 0.0 and norms[-1][1] > 0


def test_save_forward_run_hands_back_zero_absorbing_records():
    """SAVE_FORWARD: the traces are those of a plain forward run; the absorbed-
    boundary slices the host stores come back as zeros (the driver checks every
    step), since a kernel run here replays the forward field instead."""
    cfg, _ = load_golden("tromp2005_kernel")
    db = database_from_config(cfg, nstep=400)
    a, _, _ = run_forward(db)
    b, _, _ = run_forward(db, save_forward=True)
    assert np.array_equal(a, b)


def test_tromp2005_kernel_run_through_the_fortran_interface():
    """EXAMPLES/Tromp2005_kernel as SIMULATION_TYPE = 3 through
    prepare_fields_elastic_adj_dev, prepare_sim2_or_3_const_device and
    transfer_kernels_el_to_host: the adjoint traces and the kernel sums equal
    the library's own gradient run (sf2d_fwi, lambda formed in FP64 there and as
    kappa - mu in FP32 here), and the kernels scaled as
    save_adjoint_kernels.f90:134-141 scales them reach the maxima of the
    reference's kernel run."""
    import json
    import os

    from helpers import GOLDEN
    from fortran_driver import run_kernel
    from specfem2d_b200.fwi import FWIGradient
    from specfem2d_b200.setup.adjoint import cross_correlation_adjoint_source, derived_kernels

    cfg, seis = load_golden("tromp2005_kernel")
    adj_ref = dict(np.load(os.path.join(GOLDEN, "tromp2005_kernel_adjoint.npz")))
    with open(os.path.join(GOLDEN, "tromp2005_kernel_adjoint.json")) as f:
        log = json.load(f)
    traces = np.stack([seis["S0001_BXX"], seis["S0001_BXZ"]], axis=1)
    adj, _ = cross_correlation_adjoint_source(adj_ref["t_forward"], traces, 27.0, 32.0, 1)
    db = database_from_config(cfg)
    adj32 = adj.astype(np.float32).reshape(1, -1, 2)
    aseis, _, norms, kl = run_kernel(db, adj32, check_every=400)
    rs, ms, ks = kl["rho"], kl["mu"], kl["kappa"]
    g = FWIGradient(db, checkpoint_every=200)
    g.forward()
    rk, kk, mk = g.backward(adj32)
    a = g.adjoint_seismograms()
    g.close()
    assert rel_l2(aseis, a) < 1e-5
    ref = np.stack([adj_ref["S0001_BXX"], adj_ref["S0001_BXZ"]], axis=1)
    assert rel_l2(aseis[0, :, 0], ref[:, 0]) < 1e-5
    dt = np.float32(db.deltat)
    rho, kap, mu = (np.asarray(x, np.float32).reshape(-1, 5, 5) for x in (db.rhostore, db.kappastore, db.mustore))
    rho_kl, kappa_kl, mu_kl = -rho * dt * rs, -kap * dt * ks, np.float32(-2) * mu * dt * ms
    for got, want in ((rho_kl, rk), (kappa_kl, kk), (mu_kl, mk)):
        assert rel_l2(got, want) < 1e-4
    d = derived_kernels(rho_kl, kappa_kl, mu_kl, db.rhostore, db.kappastore, db.mustore)
    got = dict(rho=rho_kl.max(), kappa=kappa_kl.max(), mu=mu_kl.max(), rhop=d["rhop"].max(),
               alpha=d["alpha"].max(), beta=d["beta"].max())
    for k, v in log["kernel_max"].items():
        assert float(got[k]) == pytest.approx(v, rel=2e-5), k
    assert all(f > 0 and b == 0 for f, b in norms) and len(norms) == 8


def test_fluid_solid_kernel_run_through_the_fortran_interface():
    """EXAMPLES/LuoYang_fluid_solid_kernel as SIMULATION_TYPE = 3 through the
    fluid calls of the interface (prepare_fields_acoustic_adj_dev, the adjoint
    and replayed sources of both domains, coupling with FORWARD_OR_ADJOINT 1
    and 3, transfer_kernels_ac_to_host): the adjoint potential trace within
    1e-5 of the reference's, every kernel within the FP32 band of the library's
    own coupled gradient run (the interface forms lambda and the fluid's
    Jacobian in FP32 as the reference's GPU code does), and the ten kernel
    maxima the reference printed."""
    from helpers import load_kernel_golden
    from fortran_driver import run_kernel
    from specfem2d_b200.coupled import coupled_kernels
    from specfem2d_b200.setup.adjoint import derived_kernels

    cfg, ref, log = load_kernel_golden("luoyang_fluid_solid_kernel")
    db = database_from_config(cfg)
    adj = np.zeros((1, db.nstep, 2), np.float32)
    adj[0, :, 0] = ref["adj_source"].astype(np.float32)
    aseis, _, norms, kl = run_kernel(db, adj, check_every=800)
    lib = coupled_kernels(db, adj, checkpoint_every=200)
    assert rel_l2(aseis[0, :, 0], ref["adjoint_trace"]) < 1e-5
    assert rel_l2(aseis, lib["adj_seis"]) < 1e-5
    dt = np.float32(db.deltat)
    rho, kap, mu = (np.asarray(x, np.float32).reshape(-1, 5, 5) for x in (db.rhostore, db.kappastore, db.mustore))
    solid = ~np.asarray(db.acoustic["ispec"], dtype=bool)
    scaled = dict(rho=-rho * dt * kl["rho"], kappa=-kap * dt * kl["kappa"], mu=np.float32(-2) * mu * dt * kl["mu"])
    for k in ("rho", "kappa", "mu"):
        assert rel_l2(scaled[k][solid], lib[k][solid]) < 1e-4, k
        assert not np.any(kl[k][~solid]), k
    for k in ("rho_ac", "kappa_ac"):
        assert rel_l2(kl[k], lib[k]) < 1e-4, k
        assert not np.any(kl[k][solid]), k
    d = derived_kernels(scaled["rho"], scaled["kappa"], scaled["mu"], db.rhostore, db.kappastore, db.mustore)
    got = dict(rho=scaled["rho"].max(), kappa=scaled["kappa"].max(), mu=scaled["mu"].max(), rhop=d["rhop"].max(),
               alpha=d["alpha"].max(), beta=d["beta"].max())
    for name, v in log["kernel_max"].items():
        assert float(got[name]) == pytest.approx(v, rel=3e-5), name
    rac, kac = kl["rho_ac"], kl["kappa_ac"]
    got_ac = dict(rho=rac.max(), kappa=kac.max(), rhop=(rac + kac).max(), alpha=(np.float32(2.0) * kac).max())
    for name, v in log["acoustic_kernel_max"].items():
        assert float(got_ac[name]) == pytest.approx(v, rel=3e-5), name
    assert all(ef > 0 and eb == 0 and af > 0 and ab == 0 for (ef, eb), (af, ab) in norms)


def test_fluid_cpml_example_through_the_fortran_interface():
    """EXAMPLES/check_absolute_amplitude_of_pressure_source_seismograms_acoustic
    (fluid only, CPML on all sides, USE_TRICK_FOR_BETTER_PRESSURE) through
    prepare_PML_device and pml_boundary_acoustic_cuda: the layer's profiles as
    the reference's GPU path passes them (abs_normalized, ALPHA_MAX_PML, d0_max,
    the XZ stores) equal the set-up's to FP32 rounding, and the pressure trace
    matches the reference's REF_SEIS and the library's own run within 1e-5."""
    from specfem2d_b200.coupled import CoupledSolver

    cfg, seis = load_golden("pressure_source_acoustic")
    db = database_from_config(cfg)
    assert db.acoustic.get("use_trick")
    out, _, norms, _ = run_forward(db, check_every=500)
    assert rel_l2(out[0, :, 0], seis["S0001_PRE"]) < 1e-5
    s = CoupledSolver(db)
    ref = s.run(db.nstep)
    assert rel_l2(out, ref) < 1e-5
    assert all(a == 0.0 and b > 0 for a, b in norms)
