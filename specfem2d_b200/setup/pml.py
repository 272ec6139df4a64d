"""Host setup of the convolutional PML (CPML) absorbing layers.

Restates, for the internal (structured) mesher:

* the PML elements and their regions -- pml_init.F90:34-291: starting from
  the elements with an absorbing edge on a side, NELEM_PML_THICKNESS layers
  grow through shared corners; an element in one side's layer is CPML_X_ONLY
  (left or right) or CPML_Z_ONLY (bottom or top), in a left/right and a
  bottom/top layer CPML_XZ;
* the damping profiles -- define_PML_coefficients (pml_init.F90:550-1367)
  without PML_PARAMETER_ADJUSTMENT: d0 = -(N+1) vp_max log(R) / (2 L) per
  side and domain (N = 2, R = 0.001), d = d0 / damping_change_factor * r^N,
  K = K_MIN + (K_MAX - 1) r^N, alpha = pi f0_max (1 - r) with r the
  normalised depth into the layer, and the separation of alpha_x, alpha_z,
  beta_x, beta_z in corner elements (:1236-1350);
* the points of the outer PML edges zeroed every step
  (determine_boundary_abs_points_PML, pml_init.F90:297-420);
* the PML terms of the mass matrices (invert_mass_matrix.F90:130-255,
  :264-372): K factors and, for Newmark, the d dt/2 terms.

All profile values are double precision, as the reference stores them.
"""
from __future__ import annotations

import math

import numpy as np

from .gll import NGLL
from .mesh import IBOTTOM, ILEFT, IRIGHT, ITOP

CPML_X_ONLY, CPML_Z_ONLY, CPML_XZ = 1, 2, 3
NPOWER = 2.0
RCOEF = 0.001
f32 = np.float32


def _corners(ibool, e):
    return {int(ibool[e, 0, 0]), int(ibool[e, 0, NGLL - 1]), int(ibool[e, NGLL - 1, 0]),
            int(ibool[e, NGLL - 1, NGLL - 1])}


def pml_elements(mesh, ibool, nelem_thickness: int):
    """(is_pml (nspec,) bool, region (nspec,) int, which (4, nspec) bool per side
    IBOTTOM, IRIGHT, ITOP, ILEFT)."""
    nspec = ibool.shape[0]
    which = np.zeros((4, nspec), dtype=bool)
    corner_elems = {}
    for e in range(nspec):
        for g in _corners(ibool, e):
            corner_elems.setdefault(g, []).append(e)
    for b, side in enumerate((IBOTTOM, IRIGHT, ITOP, ILEFT)):
        for e, t in zip(mesh.abs_ispec, mesh.abs_type):
            if int(t) == side:
                which[b, int(e)] = True
        for _ in range(2, nelem_thickness + 1):
            corners = set()
            for e in np.flatnonzero(which[b]):
                corners |= _corners(ibool, e)
            grow = set()
            for g in corners:
                grow.update(corner_elems[g])
            which[b, list(grow)] = True
    is_pml = which.any(axis=0)
    region = np.zeros(nspec, dtype=np.int32)
    bot, right, top, left = which
    region[(left ^ right) & ~top & ~bot] = CPML_X_ONLY
    region[(top ^ bot) & ~left & ~right] = CPML_Z_ONLY
    region[(left ^ right) & (top ^ bot)] = CPML_XZ
    return is_pml, region, which


def pml_boundary_points(mesh, ibool, is_pml, is_acoustic):
    """Sorted global points on the outer (absorbing) edges of PML elements,
    (acoustic list, elastic list)."""
    ac, el = set(), set()
    for e, t in zip(mesh.abs_ispec, mesh.abs_type):
        e, t = int(e), int(t)
        if not is_pml[e]:
            continue
        if t == ILEFT:
            pts = [(0, j) for j in range(NGLL)]
        elif t == IRIGHT:
            pts = [(NGLL - 1, j) for j in range(NGLL)]
        elif t == IBOTTOM:
            pts = [(i, 0) for i in range(NGLL)]
        else:
            pts = [(i, NGLL - 1) for i in range(NGLL)]
        tgt = ac if is_acoustic[e] else el
        for (i, j) in pts:
            tgt.add(int(ibool[e, j, i]))
    return np.array(sorted(ac), dtype=np.int32), np.array(sorted(el), dtype=np.int32)


def pml_mass_factor(region, pml, e, newmark: bool, dto2: float):
    """Per-point K factor of PML element e (K_x, K_x K_z or K_z) and, for
    Newmark, its d dt/2 term (d_x, d_x K_z + d_z K_x or d_z, times dt/2)."""
    r = region[e]
    if r == CPML_X_ONLY:
        k = pml["K_x"][e]
        dterm = pml["d_x"][e] * dto2
    elif r == CPML_XZ:
        k = pml["K_x"][e] * pml["K_z"][e]
        dterm = (pml["d_x"][e] * pml["K_z"][e] + pml["d_z"][e] * pml["K_x"][e]) * dto2
    else:
        k = pml["K_z"][e]
        dterm = pml["d_z"][e] * dto2
    return k, (dterm if newmark else None)


def mass_entries(ibool, elems, contrib, pml_base, pml, newmark: bool, dto2: float):
    """Ordered (point, value) mass-matrix additions over ``elems`` (ascending):
    ``contrib`` (len(elems), 5, 5) for elements outside the PML; for PML
    elements ``pml_base`` (one (5, 5) block per PML element of ``elems``, in
    order: the FP32 product w w rho J or w w / kappa J) times the K factor,
    followed at the same point by its Newmark d dt/2 term.  Returns (idx, val)
    in the reference's accumulation order."""
    elems = np.asarray(elems)
    region = pml["region"]
    is_p = region[elems] > 0
    q = np.arange(NGLL * NGLL)
    idx, val, key = [], [], []
    npm = ~is_p
    if npm.any():
        e = elems[npm]
        idx.append(ibool[e].reshape(-1))
        val.append(np.asarray(contrib)[npm].reshape(-1).astype(np.float64))
        key.append((np.flatnonzero(npm)[:, None] * 100 + q[None, :] * 2).reshape(-1))
    for n, k in enumerate(np.flatnonzero(is_p)):
        e = int(elems[k])
        kf, dterm = pml_mass_factor(region, pml, e, newmark, dto2)
        b = np.asarray(pml_base[n], dtype=np.float64)
        idx.append(ibool[e].reshape(-1))
        val.append((b * kf).reshape(-1))
        key.append(k * 100 + q * 2)
        if dterm is not None:
            idx.append(ibool[e].reshape(-1))
            val.append((b * dterm).reshape(-1))
            key.append(k * 100 + q * 2 + 1)
    if not idx:
        return np.zeros(0, dtype=np.int64), np.zeros(0)
    idx = np.concatenate(idx)
    val = np.concatenate(val)
    order = np.argsort(np.concatenate(key), kind="stable")
    return idx[order], val[order]


def _side_profile(absc, thick, d0, fac, alpha_max, k_min, k_max):
    """d, K, alpha at distance ``absc`` into a layer of thickness ``thick``."""
    if absc >= 0.0:
        rn = absc / thick
        return d0 / fac * rn ** NPOWER, k_min + (k_max - 1.0) * rn ** NPOWER, alpha_max * (1.0 - rn)
    return 0.0, 1.0, 0.0


def pml_coefficients(ibool, coord, is_pml, region, rho_vpstore, rhostore, is_acoustic, f0_max: float,
                     k_min: float = 1.0, k_max: float = 1.0, damping_factor_acoustic: float = 0.5,
                     damping_factor_elastic: float = 1.0):
    """K_x, K_z, d_x, d_z, alpha_x, alpha_z per element GLL point (nspec, 5, 5) float64;
    points outside the PML hold K = 1, d = alpha = 0.  Also the normalised
    abscissae of the x and z profiles (abs_x, abs_z; 0 where none applies),
    ALPHA_MAX_PML (alpha_max) and the largest acoustic d0 over the four sides
    (d0_max_acoustic), which the GPU path of pml_init.F90:884-914 keeps."""
    nspec = ibool.shape[0]
    x, z = coord[:, 0], coord[:, 1]
    xmin, xmax, zmin, zmax = x.min(), x.max(), z.min(), z.max()
    xorigin = xmin + (xmax - xmin) / 2.0
    zorigin = zmin + (zmax - zmin) / 2.0
    ext = {k: [1.0e30, -1.0e30] for k in ("bottom", "right", "top", "left")}
    for e in np.flatnonzero(is_pml):
        zx = region[e] in (CPML_Z_ONLY, CPML_XZ)
        xx = region[e] in (CPML_X_ONLY, CPML_XZ)
        for g in ibool[e].ravel():
            xv, zv = coord[g]
            for side, ok in (("bottom", zv < zorigin and zx), ("top", zv > zorigin and zx)):
                if ok:
                    ext[side] = [min(ext[side][0], zv), max(ext[side][1], zv)]
            for side, ok in (("right", xv > xorigin and xx), ("left", xv < xorigin and xx)):
                if ok:
                    ext[side] = [min(ext[side][0], xv), max(ext[side][1], xv)]
    thick = {}
    for k, (lo, hi) in ext.items():
        t = hi - lo
        thick[k] = 0.0 if abs(t) > 1.0e30 else t
    xoriginleft = thick["left"] + xmin
    xoriginright = xmax - thick["right"]
    zoriginbottom = thick["bottom"] + zmin
    zorigintop = zmax - thick["top"]
    vpmax_ac = vpmax_el = 0.0
    for e in np.flatnonzero(is_pml):
        vp = float((rho_vpstore[e].astype(f32) / rhostore[e].astype(f32)).astype(np.float64).max())
        if is_acoustic[e]:
            vpmax_ac = max(vpmax_ac, vp)
        else:
            vpmax_el = max(vpmax_el, vp)
    alpha_max = math.pi * f0_max

    def d0(vpmax, t):
        return -(NPOWER + 1) * vpmax * math.log(RCOEF) / (2.0 * t) if t > 0.0 else 0.0

    d0s = {k: (d0(vpmax_ac, thick[k]), d0(vpmax_el, thick[k])) for k in thick}
    Kx = np.ones((nspec, NGLL, NGLL))
    Kz, dx, dz = np.ones_like(Kx), np.zeros_like(Kx), np.zeros_like(Kx)
    ax, az = np.zeros_like(Kx), np.zeros_like(Kx)
    abs_x, abs_z = np.zeros_like(Kx), np.zeros_like(Kx)
    for e in np.flatnonzero(is_pml):
        r = region[e]
        fac = damping_factor_acoustic if is_acoustic[e] else damping_factor_elastic
        dom = 0 if is_acoustic[e] else 1
        for j in range(NGLL):
            for i in range(NGLL):
                d_x = d_z = 0.0
                K_x = K_z = 1.0
                alpha_x = alpha_z = 0.0
                xv, zv = coord[ibool[e, j, i]]
                if r in (CPML_Z_ONLY, CPML_XZ):
                    for side, absc, cond in (("bottom", zoriginbottom - zv, zv < zorigin),
                                             ("top", zv - zorigintop, zv > zorigin)):
                        if cond:
                            d_z, K_z, alpha_z = _side_profile(absc, thick[side], d0s[side][dom], fac,
                                                              alpha_max, k_min, k_max)
                            if absc >= 0.0:
                                abs_z[e, j, i] = absc / thick[side]
                            if r == CPML_Z_ONLY:
                                d_x, K_x, alpha_x = 0.0, 1.0, 0.0
                if r in (CPML_X_ONLY, CPML_XZ):
                    for side, absc, cond in (("right", xv - xoriginright, xv > xorigin),
                                             ("left", xoriginleft - xv, xv < xorigin)):
                        if cond:
                            d_x, K_x, alpha_x = _side_profile(absc, thick[side], d0s[side][dom], fac,
                                                              alpha_max, k_min, k_max)
                            if absc >= 0.0:
                                abs_x[e, j, i] = absc / thick[side]
                            if r == CPML_X_ONLY:
                                d_z, K_z, alpha_z = 0.0, 1.0, 0.0
                Kx[e, j, i], Kz[e, j, i], dx[e, j, i], dz[e, j, i] = K_x, K_z, d_x, d_z
                ax[e, j, i], az[e, j, i] = alpha_x, alpha_z
    # separation of the corner parameters (pml_init.F90:1236-1350)
    dmin = 1.0e30
    for e in np.flatnonzero(is_pml):
        c = coord[ibool[e]]                                   # [j][i]
        d1 = ((c[:-1, :-1] - c[:-1, 1:]) ** 2).sum(axis=-1)   # (i, j) - (i+1, j)
        d2 = ((c[:-1, :-1] - c[1:, :-1]) ** 2).sum(axis=-1)   # (i, j) - (i, j+1)
        dmin = min(dmin, float(d1.min()), float(d2.min()))
    dmin = math.sqrt(dmin)
    sep = alpha_max / 8.0 * dmin / max(max(thick["left"], thick["right"]), max(thick["bottom"], thick["top"]))
    two = sep * 2.0
    for e in np.flatnonzero(region == CPML_XZ):
        for j in range(NGLL):
            for i in range(NGLL):
                K_x, d_x, alpha_x = Kx[e, j, i], dx[e, j, i], ax[e, j, i]
                K_z, d_z, alpha_z = Kz[e, j, i], dz[e, j, i], az[e, j, i]
                if abs(alpha_x - alpha_z) < sep:
                    if alpha_x > alpha_z:
                        alpha_x = alpha_z + two
                    else:
                        alpha_z = alpha_x + two
                beta_x = alpha_x + d_x / K_x
                if abs(beta_x - alpha_z) < sep:
                    beta_x = alpha_z + two
                beta_z = alpha_z + d_z / K_z
                if abs(beta_z - alpha_x) < sep:
                    beta_z = alpha_x + two
                dx[e, j, i] = (beta_x - alpha_x) * K_x
                dz[e, j, i] = (beta_z - alpha_z) * K_z
                ax[e, j, i], az[e, j, i] = alpha_x, alpha_z
    return dict(K_x=Kx, K_z=Kz, d_x=dx, d_z=dz, alpha_x=ax, alpha_z=az, abs_x=abs_x, abs_z=abs_z,
                alpha_max=alpha_max, d0_max_acoustic=max(v[0] for v in d0s.values()))
