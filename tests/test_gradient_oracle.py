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


def _chi(c, obs, rho_or_db, kap=None, mu=None):
    """L2 misfit of a model given as (rho, kappa, mu) or as a built Database."""
    import oracle

    d = c.db(rho_or_db, kap, mu) if kap is not None else rho_or_db
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


def _smooth_direction(c, rng):
    """A seeded smooth relative-perturbation direction (drho, dkappa, dmu): three
    Gaussians per parameter, centred away from the absorbing edges (the
    kernels are interior integrals; the Stacey terms' dependence on rho vp and
    rho vs is not part of them), amplitude 0.1."""
    out = []
    for _ in range(3):
        f = np.zeros_like(c.rho0)
        for _ in range(3):
            cx, cz, r = rng.uniform(1300.0, 2700.0), rng.uniform(900.0, 1700.0), rng.uniform(150.0, 300.0)
            f += rng.uniform(-1.0, 1.0) * np.exp(-((c.x - cx) ** 2 + (c.z - cz) ** 2) / r ** 2)
        out.append(0.1 * f / np.abs(f).max())
    return out


def test_oracle_gradient_along_ten_smooth_directions(case):
    """Ten seeded directions perturbing rho, kappa and mu together, central
    differences at eps = 1e-2 .. 1e-5.  The model is stored in CUSTOM_REAL
    (FP32) as the reference stores it, so each difference is contracted with
    the perturbation the stored model actually carries: kappa at fixed mu and
    mu at fixed lambda + 2/3 mu (the kernels' parameters).  At eps = 1e-3 and
    1e-4 the adjoint gradient and the differences agree to the consistency of
    the reference's time-paired adjoint (about 1 %, every direction within 3 %);
    the table of all four steps is printed.  At 1e-2 the misfit's curvature,
    at 1e-5 the FP32 storage of the mass matrix and boundary coefficients,
    limit the differences themselves."""
    c, obs, db0, (chi, syn, rk, kk, mk) = case
    w = db0.gll.wgll_dble
    wj = (w[None, :] * w[:, None])[None] * db0.jacobian.astype(np.float64)
    r0, k0, m0 = (a.astype(np.float64) for a in (db0.rhostore, db0.kappastore, db0.mustore))
    rng = np.random.default_rng(10)

    def model(dr, dk, dm, eps):
        m = c.mu0 * np.exp(eps * dm)
        k = (c.kappa0 - c.mu0 / 3.0 + m / 3.0) * np.exp(eps * dk)
        return c.db(c.rho0 * np.exp(eps * dr), k, m)

    table = []
    for _ in range(10):
        dr, dk, dm = _smooth_direction(c, rng)
        row = []
        for eps in (1e-2, 1e-3, 1e-4, 1e-5):
            dp, dn = model(dr, dk, dm, eps), model(dr, dk, dm, -eps)
            rp, kp, mp = (a.astype(np.float64) for a in (dp.rhostore, dp.kappastore, dp.mustore))
            rn, kn, mn = (a.astype(np.float64) for a in (dn.rhostore, dn.kappastore, dn.mustore))
            dmu = mp - mn
            g = float(np.sum(wj * (rk * (rp - rn) / r0 + kk * ((kp - kn) - dmu / 3.0) / k0 + mk * dmu / m0)))
            fd = _chi(c, obs, dp) - _chi(c, obs, dn)
            row.append(abs(g - fd) / abs(fd))
        table.append(row)
    table = np.array(table)
    print("FD relative error, rows = directions, columns = eps 1e-2 1e-3 1e-4 1e-5:")
    print(np.array2string(table, precision=2))
    assert np.all(table[:, 1:3].min(axis=1) < 3e-2)
    assert np.median(table[:, 1]) < 1.5e-2
