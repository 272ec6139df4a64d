"""The kernel run of a coupled fluid-solid mesh on the GPU (sf2d_coupled_fwi_*)
against the oracle and the reference's EXAMPLES/LuoYang_fluid_solid_kernel
run: forward potential trace, adjoint potential trace, the solid and fluid
kernels (whole arrays within the FP32 band of the FP64 oracle) and the ten
kernel maxima the reference printed.

Tolerance policy (relative L2), as for the other GPU paths: within 1e-5 of the
FP32 oracle, or at most 1.5x as far from the FP64 oracle as the FP32 oracle is."""
import numpy as np
import pytest

from helpers import load_kernel_golden, rel_l2
from specfem2d_b200.setup.adjoint import derived_kernels
from specfem2d_b200.setup.from_par_file import database_from_config

pytestmark = pytest.mark.gpu


def _close(gpu, o32, o64, factor=1.5):
    return rel_l2(gpu, o32) < 1e-5 or rel_l2(gpu, o64) < factor * rel_l2(o32, o64)


@pytest.fixture(scope="module")
def runs():
    import oracle
    from specfem2d_b200.coupled import coupled_kernels

    cfg, ref, log = load_kernel_golden("luoyang_fluid_solid_kernel")
    db = database_from_config(cfg)
    adj = np.zeros((1, db.nstep, 2))
    adj[0, :, 0] = ref["adj_source"].astype(np.float32)
    gpu = coupled_kernels(db, adj, checkpoint_every=400)
    o32 = oracle.kernels(db, adj, checkpoint_every=400, precision=4)
    o64 = oracle.kernels(db, adj, checkpoint_every=400, precision=8)
    return db, ref, log, gpu, o32, o64


def test_forward_and_adjoint_traces(runs):
    db, ref, _, gpu, o32, o64 = runs
    win = ref["t"] <= 1.274
    assert rel_l2(gpu["seis"][0, win, 0], ref["adj_source"][win]) < 5e-6
    assert _close(gpu["seis"][0, :, 0], o32["seis"][0, :, 0], o64["seis"][0, :, 0])
    assert rel_l2(gpu["adj_seis"][0, :, 0], ref["adjoint_trace"]) < 1e-5
    assert _close(gpu["adj_seis"][0, :, 0], o32["adj_seis"][0, :, 0], o64["adj_seis"][0, :, 0])


@pytest.mark.parametrize("name", ["rho", "kappa", "mu", "rho_ac", "kappa_ac"])
def test_kernels_match_the_oracle(runs, name):
    _, _, _, gpu, o32, o64 = runs
    assert _close(gpu[name], o32[name], o64[name]), name
    fluid = np.asarray(runs[0].acoustic["ispec"], dtype=bool)
    other = fluid if name in ("rho", "kappa", "mu") else ~fluid
    assert not np.any(gpu[name][other])


def test_kernel_maxima_match_ref_kernel(runs):
    db, _, log, gpu, _, _ = runs
    d = derived_kernels(gpu["rho"], gpu["kappa"], gpu["mu"], db.rhostore, db.kappastore, db.mustore)
    got = dict(rho=gpu["rho"].max(), kappa=gpu["kappa"].max(), mu=gpu["mu"].max(), rhop=d["rhop"].max(),
               alpha=d["alpha"].max(), beta=d["beta"].max())
    for name, v in log["kernel_max"].items():
        assert float(got[name]) == pytest.approx(v, rel=2e-5), name
    rac, kac = gpu["rho_ac"], gpu["kappa_ac"]
    got_ac = dict(rho=rac.max(), kappa=kac.max(), rhop=(rac + kac).max(), alpha=(np.float32(2.0) * kac).max())
    for name, v in log["acoustic_kernel_max"].items():
        assert float(got_ac[name]) == pytest.approx(v, rel=2e-5), name
