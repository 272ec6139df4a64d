"""Pins the setup + CPU oracle against the reference's own golden seismograms.

EXAMPLES/Tromp2005_kernel (elastic, Stacey on three sides, Newmark, force
source with a first-derivative-of-Gaussian time function) was run by the
reference xspecfem2D (FP32) to produce REF_SEIS/AA.S0001.BX?.semd.  The
fixtures in tests/golden were extracted from it by tests/golden/make_golden.py.
"""
import os

import numpy as np
import pytest

from helpers import initial_mode_run, load_golden, rel_l2, within_fp32_band
from specfem2d_b200.setup.from_par_file import database_from_config


@pytest.fixture(scope="module")
def tromp():
    cfg, seis = load_golden("tromp2005_kernel")
    db = database_from_config(cfg)
    return cfg, seis, db


def test_setup_matches_reference_log(tromp):
    cfg, _, db = tromp
    # locate_source / locate_receivers printed (1-based element, xi, gamma)
    (se, sxi, sg), (re_, rxi, rg) = cfg["log_locations"]
    assert db.source_ispec[0] + 1 == se and db.rec_ispec[0] + 1 == re_
    assert db.src_xi[0] == pytest.approx(sxi, abs=1e-12) and db.src_gamma[0] == pytest.approx(sg, abs=1e-12)
    assert db.rec_xi[0] == pytest.approx(rxi, abs=1e-12) and db.rec_gamma[0] == pytest.approx(rg, abs=1e-12)
    # 80 x 32 quads, NGLL = 5 -> (4*80+1) * (4*32+1) points
    assert db.nspec == 2560 and db.nglob == 321 * 129
    assert db.t0 == 8.0


def test_oracle_fp32_reproduces_ref_seis(tromp):
    import oracle

    _, seis, db = tromp
    o = oracle.Oracle(db, 4)
    out = o.run(db.nstep)
    assert rel_l2(out[0, :, 0], seis["S0001_BXX"]) < 1e-5
    assert rel_l2(out[0, :, 1], seis["S0001_BXZ"]) < 1e-5
    # trace time axis: t = (it-1) * DT - t0
    assert float(seis["t_first"]) == pytest.approx(-db.t0)
    assert float(seis["t_step"]) == pytest.approx(db.dt)


def test_oracle_fp64_close_to_fp32(tromp):
    import oracle

    _, seis, db = tromp
    o = oracle.Oracle(db, 8)
    out = o.run(db.nstep)
    # the FP64 run differs from the FP32 reference output by FP32 rounding only
    assert rel_l2(out[0, :, 0], seis["S0001_BXX"]) < 1e-4
    assert rel_l2(out[0, :, 1], seis["S0001_BXZ"]) < 1e-4


def test_oracle_thread_count_invariant(tromp):
    import oracle

    _, _, db = tromp
    a = oracle.Oracle(db, 4).run(200, nthreads=1)
    b = oracle.Oracle(db, 4).run(200, nthreads=3)
    assert np.array_equal(a, b)


def test_anisotropic_example_matches_ref_seis():
    """EXAMPLES/anisotropic_isotropic_model: a 5-element-thick anisotropic layer
    (c11 c13 c33 c55) between isotropic layers, Stacey on all sides."""
    import oracle

    cfg, seis = load_golden("anisotropic_isotropic_model")
    db = database_from_config(cfg)
    assert db.aniso is not None and int(db.aniso["ispec"].sum()) == 250
    out = oracle.Oracle(db, 4).run(db.nstep)
    assert rel_l2(out[0, :, 0], seis["S0001_BXX"]) < 1e-5
    assert rel_l2(out[0, :, 1], seis["S0001_BXZ"]) < 1e-5


def test_viscoelastic_example_matches_ref_seis_before_boundary_reflections():
    """EXAMPLES/attenuation/viscoelastic: 3 SLS, Qkappa 22.3, Qmu 20, Ricker 18 Hz.
    The reference run uses CPML; with Stacey in its place the traces agree until
    waves that touched the absorbing boundary arrive (after ~0.4 s here)."""
    import oracle

    cfg, seis = load_golden("attenuation_viscoelastic")
    db = database_from_config(cfg, absorbing_as_stacey=True)
    assert db.atten is not None
    (se, sxi, sg), (re_, rxi, rg) = cfg["log_locations"]
    assert db.source_ispec[0] + 1 == se and db.rec_ispec[0] + 1 == re_
    out = oracle.Oracle(db, 4).run(db.nstep)
    t = float(seis["t_first"]) + float(seis["t_step"]) * np.arange(db.nstep)
    w = t <= 0.4
    assert rel_l2(out[0, w, 0], seis["S0001_BXX"][w]) < 1e-5
    assert rel_l2(out[0, w, 1], seis["S0001_BXZ"][w]) < 1e-5


def test_viscoelastic_cpml_example_matches_ref_seis_full_trace():
    """The same example with its own CPML layers (3 elements, attenuating):
    pml_compute_memory_variables_viscoelastic restated in the oracle; the whole
    1400-step trace matches REF_SEIS."""
    import oracle

    cfg, seis = load_golden("attenuation_viscoelastic")
    db = database_from_config(cfg)
    assert db.pml is not None and int(np.sum(db.pml["visco"])) > 0
    out = oracle.Oracle(db, 4).run(db.nstep)
    assert rel_l2(out[0, :, 0], seis["S0001_BXX"]) < 1e-5
    assert rel_l2(out[0, :, 1], seis["S0001_BXZ"]) < 1e-5


def test_oracle_lddrk_close_to_newmark():
    """The LDDRK restatement (6 stages, update_displacement_LDDRK.F90) and the
    Newmark one solve the same problem: traces agree to time-discretisation error."""
    import oracle

    cfg, seis = load_golden("attenuation_viscoelastic")
    nm = database_from_config(cfg, absorbing_as_stacey=True)
    lk = database_from_config(cfg, absorbing_as_stacey=True, time_scheme=2)
    a = oracle.Oracle(nm, 4).run(nm.nstep)
    b = oracle.Oracle(lk, 4).run(lk.nstep)
    assert rel_l2(b, a) < 2e-2
    t = float(seis["t_first"]) + float(seis["t_step"]) * np.arange(nm.nstep)
    w = t <= 0.4
    assert rel_l2(b[0, w, 0], seis["S0001_BXX"][w]) < 2e-2


def _ocean(nstep=None, time_scheme=None):
    cfg, seis = load_golden("tomographic_ocean_model")
    t = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                             "tomographic_ocean_model_tomo.npz"))
    db = database_from_config(cfg, nstep=nstep, time_scheme=time_scheme,
                              tomo=(t["x"], t["z"], t["vp"], t["vs"], t["rho"]))
    return cfg, seis, db


OCEAN_STATIONS = (1, 3, 6, 9, 12, 14, 16, 18, 20, 22)


@pytest.fixture(scope="module")
def ocean():
    return _ocean()


def test_ocean_setup_matches_reference_log(ocean):
    """EXAMPLES/tomographic_ocean_model: 40 rows of tomographic water over 20 rows
    of rock, 80 coupling edges, 80 free-surface elements, 22 receivers."""
    cfg, _, db = ocean
    ac = db.acoustic
    assert int(ac["ispec"].sum()) == 3200 and db.nspec == 4800
    assert len(ac["cpl_ac_iglob"]) == 80 * 5 and len(ac["free_iglob"]) == 4 * 80 + 1
    locs = cfg["log_locations"]
    assert db.source_ispec[0] + 1 == locs[0][0]
    assert db.src_xi[0] == pytest.approx(locs[0][1], abs=1e-9) and db.src_gamma[0] == pytest.approx(locs[0][2], abs=1e-9)
    assert len(db.rec_ispec) == 22 == len(locs) - 1
    for r, (e, xi, g) in enumerate(locs[1:]):
        assert db.rec_ispec[r] + 1 == e
        assert db.rec_xi[r] == pytest.approx(xi, abs=1e-9) and db.rec_gamma[r] == pytest.approx(g, abs=1e-9)


def test_ocean_oracle_reproduces_ref_seis(ocean):
    """Coupled fluid-solid run: the FP32 oracle sits as close to the reference's
    FP32 traces as the FP64 oracle does (the remaining gap is FP32 rounding of
    both FP32 runs)."""
    import oracle

    _, seis, db = ocean
    o32 = oracle.Oracle(db, 4).run(db.nstep)
    o64 = oracle.Oracle(db, 8).run(db.nstep)
    got32, got64, ref = [], [], []
    for k in OCEAN_STATIONS:
        for c, ci in (("BXX", 0), ("BXZ", 1)):
            r = seis[f"S{k:04d}_{c}"]
            assert rel_l2(o32[k - 1, :, ci], r) < 2.0 * rel_l2(o64[k - 1, :, ci], r) + 2e-6
            got32.append(o32[k - 1, :, ci]); got64.append(o64[k - 1, :, ci]); ref.append(r)
    assert rel_l2(np.concatenate(got32), np.concatenate(ref)) < 3e-5
    assert rel_l2(np.concatenate(got64), np.concatenate(ref)) < 3e-5


def test_ocean_oracle_lddrk_close_to_newmark():
    """The acoustic LDDRK update (update_displacement_LDDRK.F90:88-115) with
    coupling solves the same problem as Newmark."""
    import oracle

    _, seis, nm = _ocean(nstep=900)
    _, _, lk = _ocean(nstep=900, time_scheme=2)
    a = oracle.Oracle(nm, 4).run(nm.nstep)
    b = oracle.Oracle(lk, 4).run(lk.nstep)
    assert rel_l2(b, a) < 2e-2


def test_cpml_elastic_example_matches_ref_seis():
    """EXAMPLES/semi_infinite_homogeneous: CPML layers of 3 elements on all four
    sides of an elastic square (564 PML elements, as the reference reports)."""
    import oracle

    cfg, seis = load_golden("semi_infinite_homogeneous")
    db = database_from_config(cfg)
    assert int((db.pml["region"] > 0).sum()) == 564 and len(db.stacey_iglob) == 0
    (se, sxi, sg), (re_, rxi, rg) = cfg["log_locations"]
    assert db.source_ispec[0] + 1 == se and db.rec_ispec[0] + 1 == re_
    out = oracle.Oracle(db, 4).run(db.nstep)
    assert rel_l2(out[0, :, 0], seis["S0001_BXX"]) < 1e-5
    assert rel_l2(out[0, :, 1], seis["S0001_BXZ"]) < 1e-5


@pytest.mark.parametrize("name,npml", [("force_source_elastic", 492), ("moment_tensor_dip_slip", 564)])
def test_cpml_force_and_moment_tensor_examples_match_ref_seis(name, npml):
    """EXAMPLES/check_absolute_amplitude_of_force_source_seismograms_elastic
    (vertical force at a point shared by four elements) and
    EXAMPLES/infinite_homogeneous_moment_tensor_vertical_dip_slip (moment-tensor
    source, Mxz = 1, factor 1e8), both with 3-element CPML layers: source and
    receiver elements as the reference's output.log reports them, and both
    traces over the whole run."""
    import oracle

    cfg, seis = load_golden(name)
    db = database_from_config(cfg)
    assert int((db.pml["region"] > 0).sum()) == npml
    (se, _, _), (re_, _, _) = cfg["log_locations"]
    assert db.source_ispec[0] + 1 == se and db.rec_ispec[0] + 1 == re_
    out = oracle.Oracle(db, 4).run(db.nstep)
    assert rel_l2(out[0, :, 0], seis["S0001_BXX"]) < 1e-5
    assert rel_l2(out[0, :, 1], seis["S0001_BXZ"]) < 1e-5


def test_nine_node_topography_fluid_example_matches_ref_seis():
    """EXAMPLES/simple_topography_and_also_a_simple_fluid_layer: 9-node
    (NGNOD = 9) elements under a curved surface, a fluid layer, 3-element CPML;
    the 11 stored stations over the whole run."""
    import oracle

    cfg, seis = load_golden("topography_fluid_layer")
    db = database_from_config(cfg)
    assert db.mesh.ngnod == 9 and db.acoustic is not None and db.pml is not None
    out = oracle.Oracle(db, 4).run(db.nstep)
    for k in range(11):
        for c, comp in enumerate(("BXX", "BXZ")):
            assert rel_l2(out[k, :, c], seis[f"S{k + 1:04d}_{comp}"]) < 1e-5


def test_cpml_acoustic_pressure_example_matches_ref_seis():
    """EXAMPLES/check_absolute_amplitude_of_pressure_source_seismograms_acoustic:
    fluid only, CPML on all sides (492 PML elements), Gaussian pressure source
    with USE_TRICK_FOR_BETTER_PRESSURE, one pressure receiver."""
    import oracle

    cfg, seis = load_golden("pressure_source_acoustic")
    db = database_from_config(cfg)
    assert int((db.pml["region"] > 0).sum()) == 492 and db.seismotype == 4
    out = oracle.Oracle(db, 4).run(db.nstep)
    assert rel_l2(out[0, :, 0], seis["S0001_PRE"]) < 1e-5
    assert float(seis["t_first"]) == pytest.approx(-db.t0)


def test_cpml_coupled_absorbs_like_stacey_before_reflections():
    """The coupled model with CPML instead of Stacey (the PML terms of both
    coupling directions are active where the sea floor crosses the side
    layers): the pressure traces agree until boundary waves return."""
    import oracle
    from specfem2d_b200 import configs

    st = configs.c2_coupled(nstep=700, nrec=9, scale=16)
    pm = configs.c2_coupled(nstep=700, nrec=9, scale=16, pml_thickness=3)
    assert (pm.pml["region"][pm.acoustic["ispec"]] > 0).any()
    a = oracle.Oracle(st, 4).run(st.nstep)
    b = oracle.Oracle(pm, 4).run(pm.nstep)
    w = slice(0, 500)  # direct and sea-floor waves only
    assert rel_l2(b[:, w], a[:, w]) < 5e-3


@pytest.fixture(scope="module")
def lddrk_mode():
    cfg, seis = load_golden("initial_mode_lddrk")
    db = database_from_config(cfg)
    ref = np.stack([seis["S0001_BXX"], seis["S0001_BXZ"]], axis=1)
    return cfg, db, ref, initial_mode_run(db, 4), initial_mode_run(db, 8)


def test_lddrk_initial_mode_example_matches_ref_seis(lddrk_mode):
    """EXAMPLES/initial_mode_LDDRK pins the 6-stage LDDRK scheme: a 2 km square of
    fluid (50 x 50 elements; neither Stacey nor CPML, so every edge is a free
    surface), the (2, 3) membrane mode of prepare_initial_field.F90 as initial
    potential, 5500 steps, one displacement receiver (grad chi / rho).

    REF_SEIS is an FP32 run.  Over 5500 steps its FP32 rounding moves it away
    from the FP64 solution by as much as the FP32 oracle moves from the FP64
    oracle (1.2e-3 on the small x component, 1.9e-4 on z), so the pin is that
    the reference's traces lie within that FP32 band around the FP64 oracle,
    on early and late windows; the FP32 oracle is within 2.5x that band of them."""
    cfg, db, ref, o32, o64 = lddrk_mode
    assert db.nspec == 2500 and db.nglob == 201 * 201 and db.time_scheme == 2
    assert db.acoustic["free_iglob"].size == 800 and db.source_ispec.size == 0
    assert db.rec_ispec[0] + 1 == cfg["log_locations"][0][0]
    assert db.initial_field["omega"] == pytest.approx(16.990760098708467, rel=1e-15)
    # the first recorded sample (after one step) agrees to FP32 rounding of the field
    assert rel_l2(o64[0], ref[0]) < 2e-5
    assert within_fp32_band(ref, o64, o32, o64)
    for c in (0, 1):
        assert rel_l2(o32[:, c], ref[:, c]) < 2.5 * rel_l2(o32[:, c], o64[:, c])


def test_lddrk_pin_detects_a_coefficient_slip(lddrk_mode, monkeypatch):
    """A planted mistake in the oracle (BETA_LDDRK[1] off by 1e-4 relative) moves the
    FP64 traces out of the band the reference's traces sit in."""
    import specfem2d_b200.setup.solver_setup as ss

    cfg, db, ref, o32, o64 = lddrk_mode
    beta = ss.BETA_LDDRK.copy()
    beta[1] = np.float32(beta[1] * (1.0 + 1e-4))
    monkeypatch.setattr(ss, "BETA_LDDRK", beta)
    bad = initial_mode_run(db, 8)
    assert not within_fp32_band(ref, bad, o32, o64)
