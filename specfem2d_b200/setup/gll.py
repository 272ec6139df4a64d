"""Gauss-Lobatto-Legendre quadrature and Lagrange interpolants for NGLL = 5.

Host-side setup restating, in scalar IEEE double arithmetic with the same
operation order, the reference routines:

* ``zwgljd`` / ``zwgjd`` / ``jacg`` / ``jacobf`` / ``endw1`` / ``endw2`` /
  ``pnormj`` / ``gammaf`` -- src/shared/gll_library.f90:44-597
* ``pnleg`` / ``pndleg`` -- src/shared/gll_library.f90:340-409
* ``lagrange_any`` / ``lagrange_deriv_GLL`` -- src/shared/lagrange_poly.f90:34-140
* ``define_derivation_matrices`` -- src/specfem2D/define_derivation_matrices.f90:34-90
* ``define_shape_functions`` (NGNOD = 4 and 9) -- src/shared/define_shape_functions.f90:34-140

Scalars use Python floats (C doubles) and ``math`` (the C library's
``cos``/``atan``/``sqrt``/``pow``), so the nodes, weights and hprime values
are the ones the Fortran setup produces.
"""
from __future__ import annotations

import math

import numpy as np

NGLL = 5
PI = 3.141592653589793


def _gammaf(x: float) -> float:
    # src/shared/gll_library.f90:148-172 (table of the values the code needs)
    g = 1.0
    if x == -0.5:
        g = -2.0 * math.sqrt(PI)
    if x == 0.5:
        g = math.sqrt(PI)
    if x == 1.0:
        g = 1.0
    if x == 2.0:
        g = 1.0
    if x == 1.5:
        g = math.sqrt(PI) / 2.0
    if x == 2.5:
        g = 1.5 * math.sqrt(PI) / 2.0
    if x == 3.5:
        g = 2.5 * 1.5 * math.sqrt(PI) / 2.0
    if x == 3.0:
        g = 2.0
    if x == 4.0:
        g = 6.0
    if x == 5.0:
        g = 24.0
    if x == 6.0:
        g = 120.0
    return g


def _jacobf(n: int, alp: float, bet: float, x: float):
    # src/shared/gll_library.f90:282-334; returns (poly, pder, polym1, pderm1, polym2, pderm2)
    apb = alp + bet
    poly = 1.0
    pder = 0.0
    psave = 0.0
    pdsave = 0.0
    polym1 = pderm1 = polym2 = pderm2 = 0.0
    if n == 0:
        return poly, pder, polym1, pderm1, polym2, pderm2
    polyl = poly
    pderl = pder
    poly = (alp - bet + (apb + 2.0) * x) / 2.0
    pder = (apb + 2.0) / 2.0
    if n == 1:
        return poly, pder, polym1, pderm1, polym2, pderm2
    for k in range(2, n + 1):
        dk = float(k)
        a1 = 2.0 * dk * (dk + apb) * (2.0 * dk + apb - 2.0)
        a2 = (2.0 * dk + apb - 1.0) * (alp ** 2 - bet ** 2)
        b3 = 2.0 * dk + apb - 2.0
        a3 = b3 * (b3 + 1.0) * (b3 + 2.0)
        a4 = 2.0 * (dk + alp - 1.0) * (dk + bet - 1.0) * (2.0 * dk + apb)
        polyn = ((a2 + a3 * x) * poly - a4 * polyl) / a1
        pdern = ((a2 + a3 * x) * pder - a4 * pderl + a3 * poly) / a1
        psave = polyl
        pdsave = pderl
        polyl = poly
        poly = polyn
        pderl = pder
        pder = pdern
    polym1 = polyl
    pderm1 = pderl
    polym2 = psave
    pderm2 = pdsave
    return poly, pder, polym1, pderm1, polym2, pderm2


def _jacg(np_: int, alpha: float, beta: float) -> list:
    # src/shared/gll_library.f90:178-276
    xjac = [0.0] * np_
    n = np_ - 1
    dth = 4.0 * math.atan(1.0) / (2.0 * float(n) + 2.0)
    xlast = 0.0
    for j in range(1, np_ + 1):
        if j == 1:
            x = math.cos((2.0 * (float(j) - 1.0) + 1.0) * dth)
        else:
            x1 = math.cos((2.0 * (float(j) - 1.0) + 1.0) * dth)
            x2 = xlast
            x = (x1 + x2) / 2.0
        for _ in range(10):
            p, pd, _, _, _, _ = _jacobf(np_, alpha, beta, x)
            recsum = 0.0
            for i in range(1, j):
                recsum = recsum + 1.0 / (x - xjac[np_ - i])
            delx = -p / (pd - recsum * p)
            x = x + delx
            if abs(delx) < 1.0e-12:
                break
        xjac[np_ - j] = x
        xlast = x
    # selection sort, ascending
    for i in range(np_):
        xmin = 2.0
        jmin = i
        for j in range(i, np_):
            if xjac[j] < xmin:
                xmin = xjac[j]
                jmin = j
        if jmin != i:
            xjac[i], xjac[jmin] = xjac[jmin], xjac[i]
    return xjac


def _pnormj(n: int, alpha: float, beta: float) -> float:
    # src/shared/gll_library.f90:415-451
    one, two = 1.0, 2.0
    dn = float(n)
    const = alpha + beta + one
    if n <= 1:
        prod = _gammaf(dn + alpha) * _gammaf(dn + beta)
        prod = prod / (_gammaf(dn) * _gammaf(dn + alpha + beta))
        return prod * two ** const / (two * dn + const)
    prod = _gammaf(alpha + one) * _gammaf(beta + one)
    prod = prod / (two * (one + const) * _gammaf(const + one))
    prod = prod * (one + alpha) * (two + alpha)
    prod = prod * (one + beta) * (two + beta)
    for i in range(3, n + 1):
        dindx = float(i)
        frac = (dindx + alpha) * (dindx + beta) / (dindx * (dindx + alpha + beta))
        prod = prod * frac
    return prod * two ** const / (two * dn + const)


def _zwgjd(np_: int, alpha: float, beta: float):
    # src/shared/gll_library.f90:457-519
    n = np_ - 1
    apb = alpha + beta
    if np_ == 1:
        z = [(beta - alpha) / (apb + 2.0)]
        w = [_gammaf(alpha + 1.0) * _gammaf(beta + 1.0) / _gammaf(apb + 2.0) * 2.0 ** (apb + 1.0)]
        return z, w
    z = _jacg(np_, alpha, beta)
    np1 = n + 1
    np2 = n + 2
    dnp1 = float(np1)
    dnp2 = float(np2)
    fac1 = dnp1 + alpha + beta + 1.0
    fac2 = fac1 + dnp1
    fac3 = fac2 + 1.0
    fnorm = _pnormj(np1, alpha, beta)
    rcoef = (fnorm * fac2 * fac3) / (2.0 * fac1 * dnp2)
    w = []
    for i in range(np_):
        p, pd, pm1, pdm1, pm2, pdm2 = _jacobf(np2, alpha, beta, z[i])
        w.append(-rcoef / (p * pdm1))
    return z, w


def _endw(n: int, alpha: float, beta: float, which: int) -> float:
    # src/shared/gll_library.f90:44-142 (endw1 for which=1, endw2 for which=2)
    zero, one, two, three, four = 0.0, 1.0, 2.0, 3.0, 4.0
    apb = alpha + beta
    f3 = zero
    if n == 0:
        return zero
    if which == 1:
        f1 = _gammaf(alpha + two) * _gammaf(beta + one) / _gammaf(apb + three)
    else:
        f1 = _gammaf(alpha + one) * _gammaf(beta + two) / _gammaf(apb + three)
    f1 = f1 * (apb + two) * two ** (apb + two) / two
    if n == 1:
        return f1
    if which == 1:
        fint1 = _gammaf(alpha + two) * _gammaf(beta + one) / _gammaf(apb + three)
    else:
        fint1 = _gammaf(alpha + one) * _gammaf(beta + two) / _gammaf(apb + three)
    fint1 = fint1 * two ** (apb + two)
    fint2 = _gammaf(alpha + two) * _gammaf(beta + two) / _gammaf(apb + four)
    fint2 = fint2 * two ** (apb + three)
    if which == 1:
        f2 = (-two * (beta + two) * fint1 + (apb + four) * fint2) * (apb + three) / four
    else:
        f2 = (two * (alpha + two) * fint1 - (apb + four) * fint2) * (apb + three) / four
    if n == 2:
        return f2
    for i in range(3, n + 1):
        di = float(i - 1)
        abn = alpha + beta + di
        abnn = abn + di
        a1 = -(two * (di + alpha) * (di + beta)) / (abn * abnn * (abnn + one))
        a2 = (two * (alpha - beta)) / (abnn * (abnn + two))
        a3 = (two * (abn + one)) / ((abnn + two) * (abnn + one))
        f3 = -(a2 * f2 + a1 * f1) / a3
        f1 = f2
        f2 = f3
    return f3


def zwgljd(np_: int = NGLL, alpha: float = 0.0, beta: float = 0.0):
    """GLL nodes and weights (src/shared/gll_library.f90:525-597)."""
    n = np_ - 1
    nm1 = n - 1
    z = [0.0] * np_
    w = [0.0] * np_
    if nm1 > 0:
        zi, wi = _zwgjd(nm1, alpha + 1.0, beta + 1.0)
        z[1:n] = zi
        w[1:n] = wi
    z[0] = -1.0
    z[np_ - 1] = 1.0
    if abs(alpha) < 1.0e-30 and abs(beta) < 1.0e-30:
        if np_ % 2 != 0:
            z[(np_ - 1) // 2] = 0.0
    for i in range(1, np_ - 1):
        w[i] = w[i] / (1.0 - z[i] ** 2)
    _, pd, _, _, _, _ = _jacobf(n, alpha, beta, z[0])
    w[0] = _endw(n, alpha, beta, 1) / (2.0 * pd)
    _, pd, _, _, _, _ = _jacobf(n, alpha, beta, z[np_ - 1])
    w[np_ - 1] = _endw(n, alpha, beta, 2) / (2.0 * pd)
    return z, w


def pnleg(z: float, n: int) -> float:
    # src/shared/gll_library.f90:380-409
    p1 = 1.0
    p2 = z
    p3 = p2
    for k in range(1, n):
        dk = float(k)
        p3 = ((2.0 * dk + 1.0) * z * p2 - dk * p1) / (dk + 1.0)
        p1 = p2
        p2 = p3
    return p3


def pndleg(z: float, n: int) -> float:
    # src/shared/gll_library.f90:340-374
    p1 = 1.0
    p2 = z
    p1d = 0.0
    p2d = 1.0
    p3d = 1.0
    for k in range(1, n):
        dk = float(k)
        p3 = ((2.0 * dk + 1.0) * z * p2 - dk * p1) / (dk + 1.0)
        p3d = ((2.0 * dk + 1.0) * p2 + (2.0 * dk + 1.0) * z * p2d - dk * p1d) / (dk + 1.0)
        p1 = p2
        p2 = p3
        p1d = p2d
        p2d = p3d
    return p3d


def lagrange_deriv_gll(i: int, j: int, zgll, nz: int = NGLL) -> float:
    """Derivative of the i-th Lagrange interpolant at node j (lagrange_poly.f90:102-140)."""
    degpoly = nz - 1
    if i == 0 and j == 0:
        return -float(degpoly) * (float(degpoly) + 1.0) * 0.25
    if i == degpoly and j == degpoly:
        return float(degpoly) * (float(degpoly) + 1.0) * 0.25
    if i == j:
        return 0.0
    return (pnleg(zgll[j], degpoly) / (pnleg(zgll[i], degpoly) * (zgll[j] - zgll[i]))
            + (1.0 - zgll[j] * zgll[j]) * pndleg(zgll[j], degpoly)
            / (float(degpoly) * (float(degpoly) + 1.0) * pnleg(zgll[i], degpoly)
               * (zgll[j] - zgll[i]) * (zgll[j] - zgll[i])))


def lagrange_any(xi: float, xigll) -> tuple:
    """Lagrange interpolants and derivatives at xi (lagrange_poly.f90:34-100)."""
    n = len(xigll)
    h = [0.0] * n
    hp = [0.0] * n
    for dgr in range(n):
        prod1 = 1.0
        prod2 = 1.0
        x0 = xigll[dgr]
        for i in range(n):
            if i != dgr:
                x = xigll[i]
                prod1 = prod1 * (xi - x)
                prod2 = prod2 * (x0 - x)
        prod2_inv = 1.0 / prod2
        h[dgr] = prod1 * prod2_inv
        s = 0.0
        for i in range(n):
            if i != dgr:
                prod3 = 1.0
                for j in range(n):
                    if j != dgr and j != i:
                        prod3 = prod3 * (xi - xigll[j])
                s = s + prod3
        hp[dgr] = s * prod2_inv
    return h, hp


class GLL:
    """GLL nodes/weights and derivative matrices as the solver stores them.

    ``hprime[i2, i1]`` = l'_{i1}(xi_{i2}) in FP32 and
    ``hprimewgll[i2, i1]`` = w_{i2} * hprime[i2, i1] computed in FP32,
    as define_derivation_matrices.f90:62-80 does (wxgll is cast to
    CUSTOM_REAL before the product).
    """

    def __init__(self) -> None:
        z, w = zwgljd(NGLL, 0.0, 0.0)
        # define_derivation_matrices.f90:60-61: middle node forced to exactly zero
        z[(NGLL - 1) // 2] = 0.0
        self.xigll = np.array(z, dtype=np.float64)
        self.zigll = self.xigll.copy()
        self.wgll_dble = np.array(w, dtype=np.float64)
        self.wxgll = self.wgll_dble.astype(np.float32)
        self.wzgll = self.wxgll.copy()
        hp = np.zeros((NGLL, NGLL), dtype=np.float64)
        for i1 in range(NGLL):
            for i2 in range(NGLL):
                hp[i2, i1] = lagrange_deriv_gll(i1, i2, z, NGLL)
        self.hprime_dble = hp
        self.hprime = hp.astype(np.float32)
        self.hprimewgll = (self.wxgll[:, None] * self.hprime).astype(np.float32)


def shape_functions(xi: float, gamma: float, ngnod: int):
    """Shape functions and their (xi, gamma) derivatives (define_shape_functions.f90:34-140)."""
    s, t = xi, gamma
    Q, H, ONE, TWO = 0.25, 0.5, 1.0, 2.0
    if ngnod == 4:
        sp, sm, tp, tm = s + ONE, s - ONE, t + ONE, t - ONE
        shape = [Q * sm * tm, -Q * sp * tm, Q * sp * tp, -Q * sm * tp]
        d1 = [Q * tm, -Q * tm, Q * tp, -Q * tp]
        d2 = [Q * sm, -Q * sp, Q * sp, -Q * sm]
        return shape, (d1, d2)
    if ngnod == 9:
        sp, sm, tp, tm = s + ONE, s - ONE, t + ONE, t - ONE
        s2, t2 = s * TWO, t * TWO
        ss, tt, st = s * s, t * t, s * t
        shape = [Q * sm * st * tm, Q * sp * st * tm, Q * sp * st * tp, Q * sm * st * tp,
                 H * tm * t * (ONE - ss), H * sp * s * (ONE - tt), H * tp * t * (ONE - ss),
                 H * sm * s * (ONE - tt), (ONE - ss) * (ONE - tt)]
        d1 = [Q * tm * t * (s2 - ONE), Q * tm * t * (s2 + ONE), Q * tp * t * (s2 + ONE),
              Q * tp * t * (s2 - ONE), -ONE * st * tm, H * (ONE - tt) * (s2 + ONE),
              -ONE * st * tp, H * (ONE - tt) * (s2 - ONE), -ONE * s2 * (ONE - tt)]
        d2 = [Q * sm * s * (t2 - ONE), Q * sp * s * (t2 - ONE), Q * sp * s * (t2 + ONE),
              Q * sm * s * (t2 + ONE), H * (ONE - ss) * (t2 - ONE), -ONE * st * sp,
              H * (ONE - ss) * (t2 + ONE), -ONE * st * sm, -ONE * t2 * (ONE - ss)]
        return shape, (d1, d2)
    raise ValueError("NGNOD must be either 4 or 9")
