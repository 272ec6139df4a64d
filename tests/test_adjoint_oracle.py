"""Pins the adjoint (SIMULATION_TYPE = 3) path of the oracle to the reference's
own kernel run of EXAMPLES/Tromp2005_kernel (run_this_example_kernel.sh):

* the adjoint source: the reference's tool (src/auxiliaries/adj_seismogram.f90,
  window 27-32 s, X component, Welch taper) applied to the forward REF_SEIS
  traces; its log printed the cross-correlation norm of each component and the
  solver printed the adjoint source's min/max as it read it;
* the adjoint traces: REF_KERNEL/AA.S0001.BX?.semd hold the adjoint wavefield at
  the station (write_seismograms.F90 records the adjoint field in a kernel run);
* the kernels: REF_KERNEL/output.log printed the maxima of rho, kappa, mu and of
  the derived rho', alpha, beta kernels (save_adjoint_kernels.f90:202-216).

The kernel run of the reference rebuilt the forward field backwards from saved
boundary values; the oracle replays it from checkpoints.  The maxima agree to
about 1e-6 either way, the size of FP32 rounding of the printed values.
"""
import json
import os

import numpy as np
import pytest

from helpers import GOLDEN, load_golden, load_kernel_golden, rel_l2
from specfem2d_b200.setup.adjoint import cross_correlation_adjoint_source, derived_kernels
from specfem2d_b200.setup.from_par_file import database_from_config


@pytest.fixture(scope="module")
def kernel_run():
    cfg, seis = load_golden("tromp2005_kernel")
    adj_ref = dict(np.load(os.path.join(GOLDEN, "tromp2005_kernel_adjoint.npz")))
    with open(os.path.join(GOLDEN, "tromp2005_kernel_adjoint.json")) as f:
        log = json.load(f)
    traces = np.stack([seis["S0001_BXX"], seis["S0001_BXZ"]], axis=1)
    adj, norms = cross_correlation_adjoint_source(adj_ref["t_forward"], traces, 27.0, 32.0, 1)
    db = database_from_config(cfg)
    ref = np.stack([adj_ref["S0001_BXX"], adj_ref["S0001_BXZ"]], axis=1)
    # read_adj_source stores the adjoint source in CUSTOM_REAL
    adj32 = adj.astype(np.float32).astype(np.float64).reshape(1, -1, 2)
    return db, log, adj, norms, adj32, ref


def test_adjoint_source_matches_the_reference_tool(kernel_run):
    db, log, adj, norms, adj32, _ = kernel_run
    # the tool printed N = dt sum(w s a) for BXX, BXY (no trace: 0) and BXZ
    assert norms["X"] == pytest.approx(log["norm"][0], rel=1e-14)
    assert norms["Z"] == pytest.approx(log["norm"][2], rel=1e-14)
    # the X component only (adj_comp = 1); the solver printed min/max after reading
    assert np.all(adj[:, 1] == 0.0)
    lo, hi = log["adj_min_max"]
    assert float(adj32.min()) == pytest.approx(lo, rel=2e-9)
    assert float(adj32.max()) == pytest.approx(hi, rel=2e-9)


def test_oracle_adjoint_traces_and_kernel_maxima_match_ref_kernel(kernel_run):
    import oracle

    db, log, _, _, adj32, ref = kernel_run
    runs = {p: oracle.adjoint_kernels(db, adj32, checkpoint_every=300, precision=p) for p in (4, 8)}
    a32, a64 = runs[4][1][0], runs[8][1][0]
    # adjoint traces: X (the driven component) within 1e-5; Z, two orders of magnitude
    # smaller, within the FP32 band of the FP64 oracle
    assert rel_l2(a32[:, 0], ref[:, 0]) < 1e-5
    assert rel_l2(a64[:, 0], ref[:, 0]) < 1e-5
    assert rel_l2(ref[:, 1], a64[:, 1]) < 1.5 * rel_l2(a32[:, 1], a64[:, 1])
    for p in (4, 8):
        _, _, rk, kk, mk = runs[p]
        d = derived_kernels(rk, kk, mk, db.rhostore, db.kappastore, db.mustore)
        got = dict(rho=rk.max(), kappa=kk.max(), mu=mk.max(), rhop=d["rhop"].max(), alpha=d["alpha"].max(),
                   beta=d["beta"].max())
        for k, v in log["kernel_max"].items():
            assert float(got[k]) == pytest.approx(v, rel=3e-6), (p, k)


# EXAMPLES/LuoYang_fluid_solid_kernel: a solid strip between two fluid blocks
# (9-node elements, Stacey on all sides), force source and one potential
# (seismotype 6) receiver in the fluid.  Its REF_KERNEL holds the adjoint
# source (the forward potential trace, zeroed after 1.274 s by the example's
# adj_source.f90), the adjoint run's potential trace at the station, and the
# maxima of the solid and of the fluid kernels (save_adjoint_kernels.f90:453-460).
# The adjoint run switches the domain order and the coupling terms
# (iterate_time.F90:298-327; compute_coupling_acoustic_el.f90:89-95 and
# compute_coupling_viscoelastic_ac.f90:89-93 for SIMULATION_TYPE 3).


@pytest.fixture(scope="module")
def fluid_solid():
    cfg, ref, log = load_kernel_golden("luoyang_fluid_solid_kernel")
    return database_from_config(cfg), cfg, ref, log


def test_fluid_solid_forward_potential_matches_the_adjoint_source(fluid_solid):
    """The forward potential at the station against the trace the example's
    tool copied into the adjoint source (its 1268 samples up to 1.274 s), and
    the source and station located at the element corners the log names."""
    import oracle

    db, cfg, ref, _ = fluid_solid
    assert db.seismotype == 6 and int((db.acoustic["ispec"] != 0).sum()) == 4800
    (e_s, xi_s, ga_s), (e_r, xi_r, ga_r) = cfg["log_locations"][:2]
    assert (db.source_ispec[0] + 1, db.src_xi[0], db.src_gamma[0]) == (e_s, xi_s, ga_s)
    assert (db.rec_ispec[0] + 1, db.rec_xi[0], db.rec_gamma[0]) == (e_r, xi_r, ga_r)
    win = ref["t"] <= 1.274
    assert int(win.sum()) == 1268 and np.all(ref["adj_source"][~win] == 0.0)
    for p in (4, 8):
        out = oracle.Oracle(db, p).run(db.nstep)
        assert rel_l2(out[0, win, 0], ref["adj_source"][win]) < 5e-6
        assert float(ref["t"][0]) == pytest.approx(-db.t0)


def test_fluid_solid_adjoint_trace_and_kernel_maxima_match_ref_kernel(fluid_solid):
    """Adjoint potential trace within 1e-6; the six solid and four fluid
    kernel maxima within 3e-6 of the printed values (as for Tromp2005_kernel;
    beta, a difference of two kernels, is the farthest at 2.1e-6)."""
    import oracle

    db, _, ref, log = fluid_solid
    adj = np.zeros((1, db.nstep, 2))
    # read_adj_source stores the adjoint source in CUSTOM_REAL, component 1
    adj[0, :, 0] = ref["adj_source"].astype(np.float32)
    lo, hi = log["adj_min_max"]
    assert float(adj.min()) == pytest.approx(lo, rel=1e-8) and float(adj.max()) == pytest.approx(hi, rel=1e-8)
    k = oracle.kernels(db, adj, checkpoint_every=400, precision=4)
    assert rel_l2(k["adj_seis"][0, :, 0], ref["adjoint_trace"]) < 1e-6
    d = derived_kernels(k["rho"], k["kappa"], k["mu"], db.rhostore, db.kappastore, db.mustore)
    got = dict(rho=k["rho"].max(), kappa=k["kappa"].max(), mu=k["mu"].max(), rhop=d["rhop"].max(),
               alpha=d["alpha"].max(), beta=d["beta"].max())
    for name, v in log["kernel_max"].items():
        assert float(got[name]) == pytest.approx(v, rel=3e-6), name
    rac, kac = k["rho_ac"], k["kappa_ac"]
    got_ac = dict(rho=rac.max(), kappa=kac.max(), rhop=(rac + kac).max(), alpha=(np.float32(2.0) * kac).max())
    for name, v in log["acoustic_kernel_max"].items():
        assert float(got_ac[name]) == pytest.approx(v, rel=3e-6), name
    # each domain's kernels vanish in the other domain's elements
    fluid = db.acoustic["ispec"] != 0
    assert not np.any(k["rho"][fluid]) and not np.any(rac[~fluid])
