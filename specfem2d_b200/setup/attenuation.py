"""Viscoelastic 3-SLS coefficients (host setup).

Restates, with the reference's precision mix:

* ``compute_attenuation_coeffs`` with USE_SOLVOPT = .false. (the default):
  ``classical_linear_least_squares`` / ``remplit_point`` / ``lfit_zener`` /
  ``func_zener`` / ``syst_LU`` / ``decomposition_LU`` / ``LUbksb``
  -- src/specfem2D/attenuation_model.f90:443-800, 2252-2298
* ``attenuation_model`` -- attenuation_model.f90:34-166 (f_min = f0/10,
  f_max = 10 f0; 1/tau_sigma and phi rounded to CUSTOM_REAL)
* Newmark recursive-convolution coefficients
  A = exp(-dt/(2 tau_sigma)), B = phi (1 - A) tau_sigma --
  src/specfem2D/prepare_attenuation.f90:378-396 (CUSTOM_REAL temporaries)

A point with Qkappa and Qmu both above 9998.999 has no attenuation
(prepare_attenuation.f90:341); its coefficients are left at zero, which
makes the memory variables and their stress correction vanish, as the
reference's negative-1/tau test does.
"""
from __future__ import annotations

import math
from functools import lru_cache

import numpy as np

PI = 3.141592653589793
TWO_PI = 2.0 * PI
N_SLS = 3
f32 = np.float32


def _decomposition_lu(a):
    n = len(a)
    indx = [0] * n
    d = 1.0
    eps = float(np.float32(1.0e-20))  # single-precision literal 1.e-20
    vv = [0.0] * n
    imax = 0
    for i in range(n):
        big = 0.0
        for j in range(n):
            if abs(a[i][j]) > big:
                big = abs(a[i][j])
        vv[i] = 1.0 / big
    for j in range(n):
        for i in range(j):
            s = a[i][j]
            for k in range(i):
                s = s - a[i][k] * a[k][j]
            a[i][j] = s
        big = 0.0
        for i in range(j, n):
            s = a[i][j]
            for k in range(j):
                s = s - a[i][k] * a[k][j]
            a[i][j] = s
            dum = vv[i] * abs(s)
            if dum >= big:
                big = dum
                imax = i
        if j != imax:
            for k in range(n):
                a[imax][k], a[j][k] = a[j][k], a[imax][k]
            d = -d
            vv[imax] = vv[j]
        indx[j] = imax
        if a[j][j] == 0.0:
            a[j][j] = eps
        if j != n - 1:
            dum = 1.0 / a[j][j]
            for i in range(j + 1, n):
                a[i][j] = a[i][j] * dum
    return indx


def _lubksb(a, indx, b):
    n = len(a)
    ii = -1
    for i in range(n):
        ip = indx[i]
        s = b[ip]
        b[ip] = b[i]
        if ii != -1:
            for j in range(ii, i):
                s = s - a[i][j] * b[j]
        elif s != 0.0:
            ii = i
        b[i] = s
    for i in range(n - 1, -1, -1):
        s = b[i]
        for j in range(i + 1, n):
            s = s - a[i][j] * b[j]
        b[i] = s / a[i][i]
    return b


def _func_zener(x, n, qref, point):
    out = []
    for k in range(n):
        num = x * (point[k] - x / qref)
        deno = point[k] * point[k] + x * x
        out.append(num / deno)
    return out


def _remplit_point(fmin, fmax, n):
    if n == 1:
        return [math.sqrt(fmin * fmax)]
    pts = []
    for l in range(1, n + 1):
        e = float(np.float32(np.float32(l - 1.0) / np.float32(n - 1.0)))  # default-REAL exponent
        p = (fmax / fmin) ** e
        pts.append(TWO_PI * p * fmin)
    return pts


def classical_linear_least_squares(qref, n, fmin, fmax):
    """(point, poids) of the linear Zener fit (attenuation_model.f90)."""
    m = 2 * n - 1
    point = _remplit_point(fmin, fmax, n)
    ref = 1.0 / qref
    xs = []
    for k in range(1, m + 1):
        e = float(np.float32(np.float32(k - 1.0) / np.float32(m - 1.0)))
        freq = (fmax / fmin) ** e
        freq = TWO_PI * fmin * freq
        xs.append(freq)
    covar = [[0.0] * n for _ in range(n)]
    beta = [0.0] * n
    for xk in xs:
        af = _func_zener(xk, n, qref, point)
        ym = ref
        sig2i = 1.0
        for l in range(n):
            wt = af[l] * sig2i
            for c in range(l + 1):
                covar[l][c] = covar[l][c] + wt * af[c]
            beta[l] = beta[l] + ym * wt
    for j in range(1, n):
        for k in range(j):
            covar[k][j] = covar[j][k]
    if n == 1:
        return point, [beta[0] / covar[0][0]]
    aux = [row[:] for row in covar]
    indx = _decomposition_lu(aux)
    poids = _lubksb(aux, indx, beta[:])
    return point, poids


def compute_attenuation_coeffs(n, qref, f0, fmin, fmax):
    point, poids = classical_linear_least_squares(qref, n, fmin, fmax)
    tau_sigma = [1.0 / p for p in point]
    tau_epsilon = [ts * (1.0 + n * w) for ts, w in zip(tau_sigma, poids)]
    return tau_epsilon, tau_sigma


@lru_cache(maxsize=4096)
def zener_parameters(qkappa: float, qmu: float, f0_ref: float, n: int = N_SLS):
    """FP32 (inv_tau_sigma, phi, tau_epsilon, Mu) for Qkappa (nu1) and for Qmu (nu2):
    attenuation_model.f90:147-160 (Mu = sum(tau_epsilon / tau_sigma) / N_SLS)."""
    fmin = f0_ref / 10.0
    fmax = f0_ref * 10.0
    te1, ts1 = compute_attenuation_coeffs(n, qkappa, f0_ref, fmin, fmax)
    te2, ts2 = compute_attenuation_coeffs(n, qmu, f0_ref, fmin, fmax)

    def parts(te, ts):
        s = 0.0
        for a, b in zip(te, ts):
            s = s + a / b
        itau = np.array([1.0 / t for t in ts]).astype(f32)
        phi = np.array([(1.0 - a / b) / b / s for a, b in zip(te, ts)]).astype(f32)
        return itau, phi, np.array(te).astype(f32), f32(s / n)

    return parts(te1, ts1), parts(te2, ts2)


def attenuation_model(qkappa: float, qmu: float, f0_ref: float, n: int = N_SLS):
    """FP32 (inv_tau_sigma_nu1, phi_nu1, inv_tau_sigma_nu2, phi_nu2) for one (Qkappa, Qmu)."""
    (it1, ph1, _, _), (it2, ph2, _, _) = zener_parameters(qkappa, qmu, f0_ref, n)
    return it1, ph1, it2, ph2


def newmark_coefficients(itau, phi, dt: float):
    """A = exp(-0.5 dt / tau_sigma), B = phi (1 - A) / (1/tau_sigma) with CUSTOM_REAL temporaries."""
    itau = np.asarray(itau, dtype=f32)
    phi = np.asarray(phi, dtype=f32)
    # scalar libm exp, as the Fortran runtime evaluates it
    temp = np.array([math.exp(-0.5 * float(t) * dt) for t in itau], dtype=np.float64).astype(f32)
    coef = ((1.0 - temp.astype(np.float64)) / itau.astype(np.float64)).astype(f32)
    return temp, (phi * coef).astype(f32)


def attenuation_arrays(qkappa, qmu, f0_ref: float, dt: float, no_atten_mask=None):
    """Per GLL point and SLS: Newmark (a1, b1, a2, b2) and LDDRK (itau1, phi1, itau2, phi2).

    ``qkappa``/``qmu`` are (nspec, 5, 5) arrays; points with both above
    9998.999, or flagged in ``no_atten_mask`` (PML elements), get zeros.
    """
    qk = np.asarray(qkappa, dtype=np.float64)
    qm = np.asarray(qmu, dtype=np.float64)
    shape = qk.shape + (N_SLS,)
    keys = ("a1", "b1", "a2", "b2", "itau1", "phi1", "itau2", "phi2", "teps1", "teps2")
    # Mu_nu1, Mu_nu2 per point (used by CPML layers in attenuating solids)
    out = {k: np.zeros(shape, dtype=f32) for k in keys}
    out["mu1"] = np.zeros(qk.shape, dtype=f32)
    out["mu2"] = np.zeros(qk.shape, dtype=f32)
    active = ~((qk > 9998.999) & (qm > 9998.999))
    if no_atten_mask is not None:
        active &= ~no_atten_mask
    if not active.any():
        return out
    import pandas as pd

    # distinct (Qkappa, Qmu) pairs by hashing (models hold a few of them); row 0 of
    # every table is the zero row of points without attenuation
    codes, uniq = pd.factorize((qk + 1j * qm).ravel())
    codes += 1
    codes[~active.ravel()] = 0
    tables = {k: np.zeros((len(uniq) + 1, N_SLS), dtype=f32) for k in keys}
    tables["mu1"] = np.zeros(len(uniq) + 1, dtype=f32)
    tables["mu2"] = np.zeros(len(uniq) + 1, dtype=f32)
    used = np.unique(codes)
    for c in used[used > 0]:
        qkv, qmv = float(uniq[c - 1].real), float(uniq[c - 1].imag)
        (it1, ph1, te1, m1), (it2, ph2, te2, m2) = zener_parameters(qkv, qmv, float(f0_ref))
        a1, b1 = newmark_coefficients(it1, ph1, dt)
        a2, b2 = newmark_coefficients(it2, ph2, dt)
        for k, v in (("a1", a1), ("b1", b1), ("a2", a2), ("b2", b2), ("itau1", it1), ("phi1", ph1),
                     ("itau2", it2), ("phi2", ph2), ("teps1", te1), ("teps2", te2), ("mu1", m1), ("mu2", m2)):
            tables[k][c] = v
    for k in out:
        out[k] = tables[k][codes].reshape(out[k].shape)
    return out
