"""The oracle's adjoint gradient (a restatement of SPECFEM2D's SIMULATION_TYPE = 3
kernels with undo_attenuation checkpointing) against finite differences of the
L2 waveform misfit, FP64.  Kernels are relative-perturbation kernels; mu_kl is
SPECFEM2D's derivative at fixed lambda + 2/3 mu (the 1/3 trace term of
compute_kernels.f90), so mu is perturbed that way here."""
import numpy as np
import pytest

from fwi_case import Case
from helpers import rel_l2


@pytest.fixture(scope="module")
def case():
    import oracle

    c = Case()
    obs = oracle.Oracle(c.true_db(), 8).run(c.nstep)
    db0 = c.start_db()
    grad = oracle.gradient(db0, obs, checkpoint_every=150, precision=8)
    return c, obs, db0, grad


def _chi(c, obs, rho, kap, mu):
    import oracle

    d = c.db(rho, kap, mu)
    s = oracle.Oracle(d, 8).run(d.nstep)
    return 0.5 * float(np.sum((s - obs) ** 2)) * float(d.dt)


@pytest.mark.parametrize("param", ["rho", "kappa", "mu"])
def test_oracle_gradient_matches_finite_differences(case, param):
    c, obs, db0, (chi, syn, rk, kk, mk) = case
    w = db0.gll.wgll_dble
    wj = (w[None, :] * w[:, None])[None] * db0.jacobian.astype(np.float64)
    dm = c.anomaly(2100.0, 1100.0, 250.0)
    K = {"rho": rk, "kappa": kk, "mu": mk}[param]
    g = float(np.sum(wj * K * dm))
    eps = 1e-3
    vals = []
    for s in (1, -1):
        r, k, m = c.rho0.copy(), c.kappa0.copy(), c.mu0.copy()
        if param == "rho":
            r = c.rho0 * np.exp(s * eps * dm)
        elif param == "kappa":
            k = c.kappa0 * np.exp(s * eps * dm)
        else:
            m = c.mu0 * np.exp(s * eps * dm)
            k3 = c.kappa0 - c.mu0 + 2.0 * c.mu0 / 3.0
            k = k3 - 2.0 * m / 3.0 + m
        vals.append(_chi(c, obs, r, k, m))
    fd = (vals[0] - vals[1]) / (2 * eps)
    assert abs(g - fd) / abs(fd) < 5e-3


def test_checkpoint_interval_does_not_change_kernels(case):
    import oracle

    c, obs, db0, (chi, syn, rk, kk, mk) = case
    g2 = oracle.gradient(db0, obs, checkpoint_every=400, precision=8)
    assert np.array_equal(g2[2], rk) and np.array_equal(g2[3], kk) and np.array_equal(g2[4], mk)
