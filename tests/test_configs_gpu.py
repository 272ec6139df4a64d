"""GPU parity at the sizes of the benchmark configurations (C1-C4) against the
FP32 and FP64 oracle on the same inputs.

* C1 (80 x 60 elastic, Stacey, 2000 steps, 20 receivers) in full;
* C2 (800 x 320 coupled fluid-solid, 20-element CPML, 400 pressure receivers) at
  full size over its first 1000 steps, with the bench's tile options;
* C3 (1600 x 800 viscoelastic, 3 SLS, 20.5 M points) over 100 Newmark steps and
  over 20 LDDRK steps;
* C4 (elastic gradient) at quarter scale, 4000 steps.

Tolerances (relative L2), written in each test: seismograms and wavefields
within 1e-5 of the FP32 oracle, or, where FP32 rounding dominates, at most
1.5x as far from the FP64 oracle as the FP32 oracle is.  Every test prints its
errors against both oracles (`pytest -s` shows them).
"""
import numpy as np
import pytest

from helpers import rel_l2
from specfem2d_b200 import configs

pytestmark = pytest.mark.gpu


def _report(name, **errs):
    print(f"PARITY {name}: " + ", ".join(f"{k} {v:.3e}" for k, v in errs.items()), flush=True)


def _close(gpu, o32, o64):
    return rel_l2(gpu, o32) < 1e-5 or rel_l2(gpu, o64) < 1.5 * rel_l2(o32, o64)


def test_c1_full_run():
    import oracle
    from specfem2d_b200.runtime import ElasticSolver

    db = configs.c1_homogeneous(nstep=2000, nrec=20)
    assert db.nglob == 77361
    runs = {}
    for p in (4, 8):
        o = oracle.Oracle(db, p)
        runs[p] = (o.run(db.nstep), o.displ)
    sol = ElasticSolver(db)
    s = sol.run(db.nstep)
    d, _, _ = sol.get_fields()
    (s32, d32), (s64, d64) = runs[4], runs[8]
    _report("C1 traces", gpu_vs_fp32=rel_l2(s, s32), gpu_vs_fp64=rel_l2(s, s64), fp32_vs_fp64=rel_l2(s32, s64))
    _report("C1 displ", gpu_vs_fp32=rel_l2(d, d32), gpu_vs_fp64=rel_l2(d, d64), fp32_vs_fp64=rel_l2(d32, d64))
    assert _close(s, s32, s64)
    assert _close(d, d32, d64)


def test_c2_full_size_first_1000_steps():
    """The bench's coupled CPML model and tile options (32-element solid tiles at 256
    threads, 64-element fluid tiles, 16-element solid CPML tiles at 128 threads):
    pressure traces at the 400 receivers (the direct wave arrives near step 900)
    and the potential and displacement fields after 1000 steps."""
    import oracle
    from specfem2d_b200.coupled import CoupledSolver

    db = configs.c2_coupled(nstep=1000, nrec=400, pml_thickness=20)
    assert db.nglob == 4100481
    sol = CoupledSolver(db, tile_elems=32, threads_per_block=256, fluid_tile_elems=64, pml_tile_elems=16,
                        pml_threads_per_block=128)
    s = sol.run(db.nstep)
    f = sol.get_fields()
    del sol
    ref = {}
    for p in (4, 8):
        o = oracle.Oracle(db, p)
        ref[p] = (o.run(db.nstep), o.get(oracle.POT), o.displ)
        del o
    (s32, c32, d32), (s64, c64, d64) = ref[4], ref[8]
    assert np.abs(s64).max() > 0
    _report("C2 pressure", gpu_vs_fp32=rel_l2(s, s32), gpu_vs_fp64=rel_l2(s, s64), fp32_vs_fp64=rel_l2(s32, s64))
    _report("C2 chi", gpu_vs_fp32=rel_l2(f["pot"], c32), gpu_vs_fp64=rel_l2(f["pot"], c64),
            fp32_vs_fp64=rel_l2(c32, c64))
    _report("C2 displ", gpu_vs_fp32=rel_l2(f["displ"], d32), gpu_vs_fp64=rel_l2(f["displ"], d64),
            fp32_vs_fp64=rel_l2(d32, d64))
    assert _close(s, s32, s64)
    assert _close(f["pot"], c32, c64)
    assert _close(f["displ"], d32, d64)


@pytest.mark.parametrize("scheme,nstep", [(1, 100), (2, 20)])
def test_c3_full_size_window(scheme, nstep):
    """The 1600 x 800 viscoelastic model (3 SLS, Qkappa 200, Qmu 60, moment tensor
    2 km deep): displacement field after the window (the wavefield is still near
    the source) and the surface traces."""
    import oracle
    from specfem2d_b200.runtime import ElasticSolver

    db = configs.c3_viscoelastic(nstep=nstep, time_scheme=scheme)
    assert db.nglob == 20489601
    sol = ElasticSolver(db)
    s = sol.run(db.nstep)
    d, _, _ = sol.get_fields()
    del sol
    ref = {}
    for p in (4, 8):
        o = oracle.Oracle(db, p)
        ref[p] = (o.run(db.nstep), o.displ)
        del o
    (s32, d32), (s64, d64) = ref[4], ref[8]
    name = "C3 Newmark" if scheme == 1 else "C3 LDDRK"
    _report(name + " displ", gpu_vs_fp32=rel_l2(d, d32), gpu_vs_fp64=rel_l2(d, d64), fp32_vs_fp64=rel_l2(d32, d64))
    _report(name + " traces", gpu_vs_fp32=rel_l2(s, s32), gpu_vs_fp64=rel_l2(s, s64), fp32_vs_fp64=rel_l2(s32, s64))
    assert np.abs(d64).max() > 0
    assert _close(d, d32, d64)
    assert _close(s, s32, s64)


def test_c4_quarter_scale_gradient():
    """250 x 100 elements, 4000 steps at the full-scale Courant number (dt 1.6e-3,
    6.4 s, long enough for reflections from the anomalies), observed data from
    the true model, adjoint source = residual.

    The residual is 0.14 % of the synthetics, so FP32 rounding of the synthetics
    (about 1e-6 of them) is about 1e-3 of the adjoint source and bounds any FP32
    gradient's agreement with FP64 (the FP32 oracle's own kernels sit 1e-2 from
    FP64 on such cases).  The kernel computation itself is checked at 1e-4:
    driven by the same FP64 residual, the GPU's adjoint sweep and kernel
    accumulation give rho, kappa and mu kernels within 1e-4 relative L2 of the
    FP64 oracle's.  The GPU synthetics are within 1e-5 of the FP32 oracle's."""
    import oracle
    from specfem2d_b200.fwi import FWIGradient

    db_true = configs.c4_gradient(nstep=4000, scale=4, true_model=True)
    db0 = configs.c4_gradient(nstep=4000, scale=4)
    obs = oracle.Oracle(db_true, 8).run(db0.nstep)
    syn32 = oracle.Oracle(db0, 4).run(db0.nstep)
    syn64, _, rk, kk, mk = oracle.adjoint_kernels(db0, lambda syn: syn - obs, checkpoint_every=200, precision=8)
    resid = syn64 - obs
    assert np.linalg.norm(resid) > 1e-4 * np.linalg.norm(syn64)
    g = FWIGradient(db0, checkpoint_every=200)
    syn = g.forward()
    kernels = g.backward(resid)
    g.close()
    _report("C4/4 synthetics", gpu_vs_fp32=rel_l2(syn, syn32), gpu_vs_fp64=rel_l2(syn, syn64),
            fp32_vs_fp64=rel_l2(syn32, syn64))
    assert rel_l2(syn, syn32) < 1e-5
    for name, got, want in zip(("rho", "kappa", "mu"), kernels, (rk, kk, mk)):
        err = rel_l2(got, want)
        _report(f"C4/4 {name}_kl (FP64 adjoint source)", gpu_vs_fp64=err)
        assert err < 1e-4, name
