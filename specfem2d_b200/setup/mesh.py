"""Internal mesher, global numbering and element geometry (host setup).

Restates, vectorised over elements but with the reference's per-point
operation order:

* interfaces-file structured meshing -- src/meshfem2D/meshfem2D.F90:127-156
  (raster element order, 4-node connectivity) and
  src/meshfem2D/read_mesh_files.F90:80-340 (spline interfaces, linear
  interpolation between them per layer)
* cubic splines -- src/shared/spline_routines.f90 (spline_construction,
  spline_evaluation, value_spline)
* absorbing edges -- src/meshfem2D/determine_abs_surface.f90:34-113
  plus corner detection src/specfem2D/read_mesh_databases.F90:985-1045
* global numbering -- src/specfem2D/createnum_fast.f90:34-222 followed by
  the first-touch renumbering of src/specfem2D/get_global.f90:36-98
* Jacobian and inverse mapping -- src/specfem2D/setup_mesh.F90:183-277 and
  src/specfem2D/recompute_jacobian.f90:37-170

Array convention: per-element GLL arrays have shape (nspec, NGLLZ, NGLLX),
i.e. [ispec][j][i], the same memory order as the Fortran ``(i,j,ispec)``.
Indices are 0-based here (the reference is 1-based).
"""
from __future__ import annotations

import dataclasses

import numpy as np

from .gll import GLL, NGLL, shape_functions

SMALLVALTOL = 1.0e-10
HUGEVAL = 1.0e30

# edge codes (src/shared constants IEDGE1..4 / IBOTTOM..ILEFT)
IBOTTOM, IRIGHT, ITOP, ILEFT = 1, 2, 3, 4


def spline_construction(xp, yp, tang1, tangn):
    """Second-derivative coefficients of a clamped cubic spline (spline_routines.f90)."""
    n = len(xp)
    c = [0.0] * n
    tmp = [0.0] * n
    c[0] = -1.0 / 2.0
    tmp[0] = (3.0 / (xp[1] - xp[0])) * ((yp[1] - yp[0]) / (xp[1] - xp[0]) - tang1)
    for i in range(1, n - 1):
        r = (xp[i] - xp[i - 1]) / (xp[i + 1] - xp[i - 1])
        c[i] = (r - 1.0) / (r * c[i - 1] + 2.0)
        tmp[i] = (6.0 * ((yp[i + 1] - yp[i]) / (xp[i + 1] - xp[i])
                         - (yp[i] - yp[i - 1]) / (xp[i] - xp[i - 1])) / (xp[i + 1] - xp[i - 1])
                  - (xp[i] - xp[i - 1]) / (xp[i + 1] - xp[i - 1]) * tmp[i - 1]) \
            / ((xp[i] - xp[i - 1]) / (xp[i + 1] - xp[i - 1]) * c[i - 1] + 2.0)
    c[n - 1] = ((3.0 / (xp[n - 1] - xp[n - 2])) * (tangn - (yp[n - 1] - yp[n - 2]) / (xp[n - 1] - xp[n - 2]))
                - 1.0 / 2.0 * tmp[n - 2]) / (1.0 / 2.0 * c[n - 2] + 1.0)
    for i in range(n - 2, -1, -1):
        c[i] = c[i] * c[i + 1] + tmp[i]
    return c


def value_spline(x, xp, yp, coefs):
    """Spline value, clamped to the end values outside [xp[0], xp[-1]] (spline_routines.f90)."""
    n = len(xp)
    if x < xp[0]:
        x = xp[0]
    if x > xp[n - 1]:
        x = xp[n - 1]
    lo, hi = 0, n - 1
    while hi - lo > 1:
        mid = (hi + lo + 2) // 2 - 1  # Fortran (hi+lo)/2 on 1-based indices
        if xp[mid] > x:
            hi = mid
        else:
            lo = mid
    if xp[hi] == xp[lo]:
        raise ValueError("incorrect interval found in spline evaluation")
    c1 = (xp[hi] - x) / (xp[hi] - xp[lo])
    c2 = (x - xp[lo]) / (xp[hi] - xp[lo])
    return (c1 * yp[lo] + c2 * yp[hi]
            + ((c1 ** 3 - c1) * coefs[lo] + (c2 ** 3 - c2) * coefs[hi]) * ((xp[hi] - xp[lo]) ** 2) / 6.0)


def read_interfaces_file(path):
    """Parse an interfaces file: returns (list of (x[], z[]) interfaces, nz per layer)."""
    toks = []
    with open(path) as f:
        for line in f:
            s = line.strip()
            if not s or s.startswith("#"):
                continue
            toks.extend(s.split())
    it = iter(toks)
    nint = int(next(it))
    interfaces = []
    for _ in range(nint):
        npt = int(next(it))
        xs, zs = [], []
        for _ in range(npt):
            xs.append(float(next(it).replace("d", "e").replace("D", "e")))
            zs.append(float(next(it).replace("d", "e").replace("D", "e")))
        interfaces.append((xs, zs))
    nz_layer = [int(next(it)) for _ in range(nint - 1)]
    return interfaces, nz_layer


@dataclasses.dataclass
class Mesh:
    """Element connectivity and coordinates as the solver sees them."""

    nspec: int
    ngnod: int
    knods: np.ndarray          # (nspec, ngnod) int, 0-based control-node ids
    coorg: np.ndarray          # (npgeo, 2) float64 control-node coordinates
    nx: int = 0
    nz: int = 0
    # absorbing edges, in the order the mesher writes them
    abs_ispec: np.ndarray = None   # (nabs,) 0-based element
    abs_type: np.ndarray = None    # (nabs,) IBOTTOM/IRIGHT/ITOP/ILEFT
    abs_corner: np.ndarray = None  # (nabs, 4) bool codeabs_corner
    free_top: bool = True
    absorb: tuple = (True, True, False, True)  # (bottom, right, top, left) outer edges absorbing
    # listed acoustic free-surface edges of an external mesh: (nfree, 5) int,
    # rows (element, imin, imax, jmin, jmax) 0-based; None on the structured mesh
    free_edges: np.ndarray = None

    def __getstate__(self):
        # the node-interpolation cache is derived data: rebuilt on demand, never pickled
        state = dict(self.__dict__)
        state.pop("_interp_cache", None)
        return state


def internal_mesh(xmin, xmax, nx, interfaces, nz_layer, absorb=(True, True, False, True),
                  ngnod=4, topography_fn=None):
    """Structured interfaces mesh (read_mesh_files.F90:80-340, meshfem2D.F90:127-156).

    ``absorb`` = (bottom, right, top, left).  ``topography_fn`` is an optional
    analytic top surface x -> z used instead of a spline of the top
    interface (for synthetic sinusoidal topography).
    """
    if ngnod not in (4, 9):
        raise ValueError("NGNOD must be either 4 or 9")
    # 9-node elements: the same grid at twice the resolution, every layer's
    # element count doubled (read_parameter_file.F90:103-108)
    mult = 1 if ngnod == 4 else 2
    nx_el, nz_el = nx, int(sum(nz_layer))
    nx = nx * mult
    nz_layer = [int(n) * mult for n in nz_layer]
    nzt = int(sum(nz_layer))
    gx = np.zeros((nx + 1, nzt + 1))
    gz = np.zeros((nx + 1, nzt + 1))
    xb, zb = interfaces[0]
    ioffset = 0
    for ilayer, nzl in enumerate(nz_layer):
        xt, zt = interfaces[ilayer + 1]
        t1 = (zb[1] - zb[0]) / (xb[1] - xb[0])
        tn = (zb[-1] - zb[-2]) / (xb[-1] - xb[-2])
        cb = spline_construction(xb, zb, t1, tn)
        t1 = (zt[1] - zt[0]) / (xt[1] - xt[0])
        tn = (zt[-1] - zt[-2]) / (xt[-1] - xt[-2])
        ct = spline_construction(xt, zt, t1, tn)
        last = ilayer == len(nz_layer) - 1
        for ix in range(nx + 1):
            absx = xmin + (xmax - xmin) * float(ix) / float(nx)
            bot0 = value_spline(absx, xb, zb, cb)
            if last and topography_fn is not None:
                top0 = float(topography_fn(absx))
            else:
                top0 = value_spline(absx, xt, zt, ct)
            for iz in range(nzl + 1):
                gamma = float(iz) / float(nzl)
                a00 = 1.0 - gamma
                a01 = gamma
                gx[ix, iz + ioffset] = absx
                gz[ix, iz + ioffset] = a00 * bot0 + a01 * top0
        ioffset += nzl
        xb, zb = xt, zt
    coorg = np.zeros(((nx + 1) * (nzt + 1), 2))
    jj, ii = np.meshgrid(np.arange(nzt + 1), np.arange(nx + 1), indexing="ij")
    ii, jj = ii.ravel(), jj.ravel()
    num = _num_9(ii, jj, nx_el, nz_el) if ngnod == 9 else jj * (nx + 1) + ii
    coorg[num, 0] = gx[ii, jj]
    coorg[num, 1] = gz[ii, jj]
    # elements in raster order, j (z) outer, i (x) inner; corners counter-clockwise
    # from bottom left, then (9 nodes) the bottom, right, top, left edge middles
    # and the centre (meshfem2D.F90:132-156)
    ej, ei = np.meshgrid(np.arange(nz_el), np.arange(nx_el), indexing="ij")
    ej, ei = ej.ravel(), ei.ravel()
    if ngnod == 4:
        knods = np.stack([ej * (nx + 1) + ei, ej * (nx + 1) + ei + 1,
                          (ej + 1) * (nx + 1) + ei + 1, (ej + 1) * (nx + 1) + ei], axis=1)
    else:
        gi, gj = 2 * ei, 2 * ej
        knods = np.stack([_num_9(gi + a, gj + b, nx_el, nz_el)
                          for a, b in ((0, 0), (2, 0), (2, 2), (0, 2), (1, 0), (2, 1), (1, 2), (0, 1), (1, 1))],
                         axis=1)
    mesh = Mesh(nspec=nx_el * nz_el, ngnod=ngnod, knods=knods.astype(np.int64), coorg=coorg, nx=nx_el, nz=nz_el)
    _absorbing_edges(mesh, absorb)
    mesh.free_top = not absorb[2]
    mesh.absorb = tuple(bool(a) for a in absorb)
    return mesh


def _num_9(i, j, nx, nz):
    """0-based control-node id of the point (i, j) of the double-resolution grid
    of a 9-node mesh with nx x nz elements (num_9, get_node_number.f90:65-83):
    corners first, then the horizontal edge middles, then the rows of vertical
    edge middles and centres."""
    i, j = np.asarray(i), np.asarray(j)
    corner = (i % 2 == 0) & (j % 2 == 0)
    even_row = (j % 2 == 0)
    n_corner = (nx + 1) * (nz + 1)
    return np.where(corner, j // 2 * (nx + 1) + i // 2,
                    np.where(even_row, n_corner + j // 2 * nx + (i + 1) // 2 - 1,
                             n_corner + nx * (nz + 1) + j // 2 * (2 * nx + 1) + i))


def _absorbing_edges(mesh: Mesh, absorb) -> None:
    """Absorbing edge list in mesher order (determine_abs_surface.f90) + corner flags."""
    ab, ar, at, al = absorb
    nx, nz = mesh.nx, mesh.nz
    isp, typ = [], []
    for iz in range(1, nz + 1):
        for ix in range(1, nx + 1):
            e = (iz - 1) * nx + ix - 1
            if ab and iz == 1:
                isp.append(e); typ.append(IBOTTOM)
            if ar and ix == nx:
                isp.append(e); typ.append(IRIGHT)
            if at and iz == nz:
                isp.append(e); typ.append(ITOP)
            if al and ix == 1:
                isp.append(e); typ.append(ILEFT)
    isp = np.array(isp, dtype=np.int64)
    typ = np.array(typ, dtype=np.int64)
    corner = absorbing_corners(isp, typ)
    mesh.abs_ispec, mesh.abs_type, mesh.abs_corner = isp, typ, corner


def absorbing_corners(isp, typ):
    """codeabs_corner of each absorbing entry: a bottom (top) edge of an element
    that also lists a left or right absorbing edge skips that corner point
    (read_mesh_databases.F90:985-1030).  Returns (nabs, 4) bool: bottom-left,
    bottom-right, top-left, top-right."""
    corner = np.zeros((len(isp), 4), dtype=bool)
    by_elem = {}
    for k, (e, t) in enumerate(zip(isp, typ)):
        by_elem.setdefault(int(e), []).append((k, int(t)))
    for k, (e, t) in enumerate(zip(isp, typ)):
        others = [tt for (kk, tt) in by_elem[int(e)] if kk != k]
        if t == IBOTTOM:
            corner[k, 0] = ILEFT in others
            corner[k, 1] = IRIGHT in others
        if t == ITOP:
            corner[k, 2] = ILEFT in others
            corner[k, 3] = IRIGHT in others
    return corner


def _shape_tables(gll: GLL, ngnod: int):
    """shape2D(in, i, j) and dershape2D at the GLL nodes: arrays [j][i][in]."""
    sh = np.zeros((NGLL, NGLL, ngnod))
    d1 = np.zeros((NGLL, NGLL, ngnod))
    d2 = np.zeros((NGLL, NGLL, ngnod))
    for j in range(NGLL):
        for i in range(NGLL):
            s, (a, b) = shape_functions(gll.xigll[i], gll.zigll[j], ngnod)
            sh[j, i] = s
            d1[j, i] = a
            d2[j, i] = b
    return sh, d1, d2


def _interp_nodes(mesh: Mesh, tab):
    """Sum_in tab[j,i,in] * coorg[knods[e,in]] accumulated in node order, for x and z.
    The result is kept on the mesh for later calls with the same table."""
    cache = mesh.__dict__.setdefault("_interp_cache", {})
    key = (tab.shape, tab.tobytes())
    if key in cache:
        return cache[key]
    xe = mesh.coorg[mesh.knods, 0]  # (nspec, ngnod)
    ze = mesh.coorg[mesh.knods, 1]
    x = np.zeros((mesh.nspec, NGLL, NGLL))
    z = np.zeros((mesh.nspec, NGLL, NGLL))
    for ia in range(mesh.ngnod):
        x += tab[None, :, :, ia] * xe[:, ia, None, None]
        z += tab[None, :, :, ia] * ze[:, ia, None, None]
    x.flags.writeable = False
    z.flags.writeable = False
    cache[key] = (x, z)
    return x, z


def createnum_fast(mesh: Mesh, gll: GLL):
    """Global numbering by coordinate sorting (createnum_fast.f90:34-222).

    Returns ibool (nspec,5,5) with ids in the sort-segment numbering, and nglob.
    Points merge when consecutive sorted coordinates differ by at most
    SMALLVALTOL times the smallest element extent, exactly as in the reference.
    """
    sh, _, _ = _shape_tables(gll, mesh.ngnod)
    xp, yp = _interp_nodes(mesh, sh)
    xp = xp.ravel()
    yp = yp.ravel()
    ntot = xp.size
    xe = xp.reshape(mesh.nspec, -1)
    ye = yp.reshape(mesh.nspec, -1)
    xtypdist = min(float((xe.max(1) - xe.min(1)).min()), float((ye.max(1) - ye.min(1)).min()), HUGEVAL)
    xtol = SMALLVALTOL * xtypdist
    o1 = np.argsort(xp, kind="stable")
    xs = xp[o1]
    brk = np.empty(ntot, dtype=bool)
    brk[0] = True
    brk[1:] = np.abs(np.diff(xs)) > xtol
    xseg = np.cumsum(brk)
    ys = yp[o1]
    o2 = np.lexsort((ys, xseg))
    ys2 = ys[o2]
    xseg2 = xseg[o2]
    brk2 = np.empty(ntot, dtype=bool)
    brk2[0] = True
    brk2[1:] = (xseg2[1:] != xseg2[:-1]) | (np.abs(np.diff(ys2)) > xtol)
    gid = np.cumsum(brk2) - 1
    iglob = np.empty(ntot, dtype=np.int64)
    iglob[o1[o2]] = gid
    return iglob.reshape(mesh.nspec, NGLL, NGLL), int(gid[-1] + 1)


def get_global(ibool):
    """First-touch renumbering in element order (get_global.f90:36-98)."""
    flat = ibool.ravel()
    uniq, first = np.unique(flat, return_index=True)
    rank = np.empty(uniq.size, dtype=np.int64)
    rank[np.argsort(first, kind="stable")] = np.arange(uniq.size)
    lut = np.empty(int(uniq.max()) + 1, dtype=np.int64)
    lut[uniq] = rank
    return lut[flat].reshape(ibool.shape)


def setup_mesh_coordinates(mesh: Mesh, gll: GLL, ibool, nglob):
    """xix, xiz, gammax, gammaz, jacobian (FP32) and coord (FP64) (setup_mesh.F90:183-277)."""
    sh, d1, d2 = _shape_tables(gll, mesh.ngnod)
    x, z = _interp_nodes(mesh, sh)
    xxi, zxi = _interp_nodes(mesh, d1)
    xgamma, zgamma = _interp_nodes(mesh, d2)
    jac = xxi * zgamma - xgamma * zxi
    if np.any(jac <= 0.0):
        bad = int(np.argwhere((jac <= 0.0).reshape(mesh.nspec, -1).any(1))[0, 0])
        raise ValueError(f"negative 2D Jacobian in element {bad + 1}")
    xix = zgamma / jac
    gammax = -zxi / jac
    xiz = -xgamma / jac
    gammaz = xxi / jac
    # coord(:, iglob): the last element visiting a point writes it
    flat = ibool.ravel()
    last = np.empty(nglob, dtype=np.int64)
    last[flat] = np.arange(flat.size)  # numpy keeps the last of repeated indices
    coord = np.stack([x.ravel()[last], z.ravel()[last]], axis=1)
    f32 = np.float32
    return dict(xix=xix.astype(f32), xiz=xiz.astype(f32), gammax=gammax.astype(f32),
                gammaz=gammaz.astype(f32), jacobian=jac.astype(f32), coord=coord,
                xstore=x, zstore=z)


def recompute_jacobian(mesh: Mesh, ispec: int, xi: float, gamma: float):
    """Scalar point mapping at (xi, gamma) in element ispec (recompute_jacobian.f90:37-170)."""
    shape, (d1, d2) = shape_functions(xi, gamma, mesh.ngnod)
    x = z = xxi = zxi = xgamma = zgamma = 0.0
    for ia in range(mesh.ngnod):
        nnum = mesh.knods[ispec, ia]
        xe = float(mesh.coorg[nnum, 0])
        ze = float(mesh.coorg[nnum, 1])
        x = x + shape[ia] * xe
        z = z + shape[ia] * ze
        xxi = xxi + d1[ia] * xe
        zxi = zxi + d1[ia] * ze
        xgamma = xgamma + d2[ia] * xe
        zgamma = zgamma + d2[ia] * ze
    jac = xxi * zgamma - xgamma * zxi
    if jac <= 0.0:
        raise ValueError(f"negative 2D Jacobian in element {ispec + 1}")
    return x, z, zgamma / jac, -xgamma / jac, -zxi / jac, xxi / jac, jac
