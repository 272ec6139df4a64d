"""Host setup of the acoustic (fluid) domain and of fluid-solid coupling.

Restates, for the potential formulation u = grad(chi) / rho of SPECFEM2D:

* element domain flags -- get_simulation_domains.f90:130-160 (an element is
  acoustic when its shear velocity is below TINYVAL);
* fluid-solid coupling edges -- repartition_coupling.f90:38-106 (pairs of an
  acoustic and an elastic element sharing an edge, acoustic elements in
  increasing order), get_coupling_edges.f90:34-125 (edge ids, ivalue/jvalue
  tables) and the per-point normals and weights of
  compute_coupling_acoustic_el.f90:36-283 and
  compute_coupling_viscoelastic_ac.f90:36-258;
* acoustic absorbing points -- compute_stacey_acoustic.f90:34-199, with the
  points shared with a coupling edge left out
  (get_coupling_edges.f90:525-570);
* the acoustic mass matrix -- invert_mass_matrix.F90:374-430 (no PML) and
  :700-790 (Newmark Stacey term), inverted as in :798-849;
* the acoustic free surface -- determine_acoustic_surface.f90:36-140 (outer
  edges of acoustic elements on non-absorbing sides) as zeroed by
  enforce_acoustic_free_surface.f90:35-96.

All per-point arithmetic is FP32 (CUSTOM_REAL) in the reference's order.
"""
from __future__ import annotations

import numpy as np

from .gll import NGLL
from .mesh import IBOTTOM, ILEFT, IRIGHT, ITOP

f32 = np.float32
TINYVAL = 1.0e-9
L = NGLL - 1

# edge traversal (0-based): begin and end corner of each edge, counter-clockwise
_BEGIN = {IBOTTOM: (0, 0), IRIGHT: (L, 0), ITOP: (L, L), ILEFT: (0, L)}
_END = {IBOTTOM: (L, 0), IRIGHT: (L, L), ITOP: (0, L), ILEFT: (0, 0)}


def _ivalue(p, edge):
    """(i, j) of point p along `edge` (ivalue/jvalue of get_coupling_edges.f90:91-110)."""
    return {IBOTTOM: (p, 0), IRIGHT: (L, p), ITOP: (L - p, L), ILEFT: (0, L - p)}[edge]


def _ivalue_inverse(p, edge):
    """(i, j) of point p along `edge` traversed backwards (ivalue_inverse/jvalue_inverse)."""
    return {IBOTTOM: (L - p, 0), IRIGHT: (L, L - p), ITOP: (p, L), ILEFT: (0, p)}[edge]


def acoustic_element_flags(vs) -> np.ndarray:
    """(nspec,) bool: acoustic when vs < TINYVAL (tested at the element's first point)."""
    vs = np.asarray(vs, dtype=np.float64)
    return vs.reshape(vs.shape[0], -1)[:, 0] < TINYVAL


def _edge_normal(geo, e, i, j, edge, gll):
    """Outward unit normal and 1-D weight at (i, j) on `edge` of element e, FP32
    (compute_coupling_acoustic_el.f90:161-230)."""
    jac = geo["jacobian"][e, j, i]
    if edge in (ITOP, IBOTTOM):
        xxi = f32(geo["gammaz"][e, j, i] * jac)
        zxi = f32(-geo["gammax"][e, j, i] * jac)
        j1d = f32(np.sqrt(f32(f32(xxi * xxi) + f32(zxi * zxi))))
        if edge == ITOP:
            nx, nz = f32(-zxi / j1d), f32(xxi / j1d)
        else:
            nx, nz = f32(zxi / j1d), f32(-xxi / j1d)
        w = f32(j1d * gll.wxgll[i])
    else:
        xgamma = f32(-geo["xiz"][e, j, i] * jac)
        zgamma = f32(geo["xix"][e, j, i] * jac)
        j1d = f32(np.sqrt(f32(f32(xgamma * xgamma) + f32(zgamma * zgamma))))
        if edge == ILEFT:
            nx, nz = f32(-zgamma / j1d), f32(xgamma / j1d)
        else:
            nx, nz = f32(zgamma / j1d), f32(-xgamma / j1d)
        w = f32(j1d * gll.wzgll[j])
    return nx, nz, w


def coupling_edges(ibool, is_acoustic):
    """Fluid-solid edges as (acoustic element, acoustic edge, elastic element,
    elastic edge), acoustic elements in increasing order, then elastic ones."""
    corner = {}
    for e in np.flatnonzero(~is_acoustic):
        for edge in (IBOTTOM, IRIGHT, ITOP, ILEFT):
            b, t = _BEGIN[edge], _END[edge]
            key = (int(ibool[e, b[1], b[0]]), int(ibool[e, t[1], t[0]]))
            corner[key] = (int(e), edge)
    out = []
    for ea in np.flatnonzero(is_acoustic):
        found = []
        for edge_a in (IBOTTOM, IRIGHT, ITOP, ILEFT):
            b, t = _BEGIN[edge_a], _END[edge_a]
            # the elastic element runs the shared edge the other way round
            hit = corner.get((int(ibool[ea, t[1], t[0]]), int(ibool[ea, b[1], b[0]])))
            if hit is not None:
                found.append((hit[0], int(ea), edge_a, hit[1]))
        for ee, ea_, edge_a, edge_e in sorted(found):
            out.append((ea_, edge_a, ee, edge_e))
    return out


def coupling_points(edges, ibool, geo, gll):
    """Per-point lists for both coupling directions, in the reference's visit order.

    acoustic side (compute_coupling_acoustic_el.f90): chi_dd[g] += w * (u . n)
    elastic side (compute_coupling_viscoelastic_ac.f90): a[g] += (w n) * (-chi_dd[g])
    Both read and write the same global point (one numbering for both
    domains); the normal is the acoustic element's outward normal.
    The fifth entry of each list is the element GLL point (ispec*25 + j*5 + i)
    of the other domain's element at that point, whose CPML profile the
    coupling uses when that element lies in a PML layer.
    """
    ac = {k: [] for k in ("iglob", "nx", "nz", "w", "pt")}
    el = {k: [] for k in ("iglob", "nx", "nz", "w", "pt")}
    for (ea, edge_a, ee, edge_e) in edges:
        for p in range(NGLL):
            ie, je = _ivalue_inverse(p, edge_e)
            ia, ja = _ivalue(p, edge_a)
            g = int(ibool[ea, ja, ia])
            if int(ibool[ee, je, ie]) != g:
                raise ValueError("fluid/solid coupling points do not match")
            nx, nz, w = _edge_normal(geo, ea, ia, ja, edge_a, gll)
            for k, v in zip(("iglob", "nx", "nz", "w", "pt"), (g, nx, nz, w, ee * 25 + je * NGLL + ie)):
                ac[k].append(v)
        for p in range(NGLL):
            ia, ja = _ivalue_inverse(p, edge_a)
            ie, je = _ivalue(p, edge_e)
            g = int(ibool[ee, je, ie])
            if int(ibool[ea, ja, ia]) != g:
                raise ValueError("fluid/solid coupling points do not match")
            nx, nz, w = _edge_normal(geo, ea, ia, ja, edge_a, gll)
            for k, v in zip(("iglob", "nx", "nz", "w", "pt"), (g, nx, nz, w, ea * 25 + ja * NGLL + ia)):
                el[k].append(v)

    def pack(d):
        return (np.array(d["iglob"], dtype=np.int32), np.array(d["nx"], dtype=f32),
                np.array(d["nz"], dtype=f32), np.array(d["w"], dtype=f32), np.array(d["pt"], dtype=np.int64))

    return pack(ac), pack(el)


def absorbing_ranges(mesh, edges):
    """Per absorbing face: the GLL (i, j) points visited by the Stacey loops.

    Bottom/top edges skip the corners shared with a left/right absorbing edge
    (codeabs_corner); edges of an acoustic element that also carries a
    coupling edge skip the point shared with it (get_coupling_edges.f90:525-570).
    """
    coupled = {}
    for (ea, edge_a, _, _) in edges:
        coupled.setdefault(ea, set()).add(edge_a)
    out = []
    for k in range(len(mesh.abs_ispec)):
        e = int(mesh.abs_ispec[k])
        t = int(mesh.abs_type[k])
        c = coupled.get(e, set())
        if t in (ILEFT, IRIGHT):
            jb = 1 if IBOTTOM in c else 0
            je = L - 1 if ITOP in c else L
            i = 0 if t == ILEFT else L
            pts = [(i, j) for j in range(jb, je + 1)]
        else:
            ib = 1 if (ILEFT in c or (mesh.abs_corner[k, 0 if t == IBOTTOM else 2])) else 0
            ie = L - 1 if (IRIGHT in c or (mesh.abs_corner[k, 1 if t == IBOTTOM else 3])) else L
            j = 0 if t == IBOTTOM else L
            pts = [(i, j) for i in range(ib, ie + 1)]
        out.append((k, e, t, pts))
    return out


def stacey_acoustic_points(mesh, geo, mat, ibool, gll, is_acoustic, edges):
    """Per absorbing GLL point of an acoustic element: iglob, weight, rho*vp
    (compute_stacey_acoustic.f90:78-180)."""
    g_l, w_l, r_l = [], [], []
    if mesh.abs_ispec is None:
        return np.zeros(0, np.int32), np.zeros(0, f32), np.zeros(0, f32)
    for (k, e, t, pts) in absorbing_ranges(mesh, edges):
        if not is_acoustic[e]:
            continue
        for (i, j) in pts:
            _, _, w = _edge_normal(geo, e, i, j, t, gll)
            g_l.append(int(ibool[e, j, i]))
            w_l.append(w)
            r_l.append(mat["rho_vpstore"][e, j, i])
    return np.array(g_l, dtype=np.int32), np.array(w_l, dtype=f32), np.array(r_l, dtype=f32)


def mass_matrix_acoustic(ibool, nglob, geo, mat, gll, is_acoustic, st_ac, newmark: bool, dt: float, pml=None):
    """rmass_inverse_acoustic (nglob,) f32: sum of w_i w_j J / kappa over acoustic
    elements, plus dt/2 * weight / (rho vp) at Newmark absorbing points; zero
    sums become 1 before inversion (invert_mass_matrix.F90:374-430, 700-790, 828-844)."""
    from .solver_setup import _sequential_f32_accumulate

    wxwz = (gll.wxgll[None, :] * gll.wzgll[:, None]).astype(f32)
    el = np.flatnonzero(is_acoustic)
    contrib = (wxwz[None].astype(f32) * geo["jacobian"][el].astype(f32)).astype(f32)
    contrib = (contrib / mat["kappastore"][el].astype(f32)).astype(f32)
    if pml is not None:
        from .pml import mass_entries

        # PML elements: w w / kappa J in that order, times K (and d dt/2), invert_mass_matrix.F90:264-372
        base = ((wxwz[None] / mat["kappastore"][el].astype(f32)).astype(f32) * geo["jacobian"][el].astype(f32)).astype(f32)
        base = base[pml["region"][el] > 0]
        idx, val = mass_entries(ibool, el, contrib, base, pml, newmark, float(f32(0.5 * float(f32(dt)))))
        m = _sequential_f32_accumulate(nglob, idx.astype(np.int64), val)
    else:
        m = _sequential_f32_accumulate(nglob, ibool[el].ravel().astype(np.int64), contrib.ravel().astype(np.float64))
    if newmark and len(st_ac[0]):
        dto2 = f32(0.5 * float(f32(dt)))
        g, w, rvp = st_ac
        for p in range(len(g)):
            m[g[p]] = f32(m[g[p]] + f32(f32(dto2 * w[p]) / rvp[p]))
    m = np.where(m <= 0, f32(1.0), m).astype(f32)
    return (f32(1.0) / m).astype(f32)


def structured_free_edges(mesh, is_acoustic):
    """(nfree, 5) rows (element, imin, imax, jmin, jmax): the outer edges of
    fluid elements on the non-absorbing sides of the structured mesh, top,
    bottom, left, right (determine_acoustic_surface.f90:50-140)."""
    nx, nz = mesh.nx, mesh.nz
    ab, ar, at, al = mesh.absorb
    rows = []
    span = {ITOP: (0, L, L, L), IBOTTOM: (0, L, 0, 0), ILEFT: (0, 0, 0, L), IRIGHT: (L, L, 0, L)}

    def add(e, edge):
        if is_acoustic[e]:
            rows.append((e,) + span[edge])

    if not at:
        for ix in range(nx):
            add((nz - 1) * nx + ix, ITOP)
    if not ab:
        for ix in range(nx):
            add(ix, IBOTTOM)
    if not al:
        for iz in range(nz):
            add(iz * nx, ILEFT)
    if not ar:
        for iz in range(nz):
            add(iz * nx + nx - 1, IRIGHT)
    return np.array(rows, dtype=np.int64).reshape(-1, 5)


def free_surface_points(mesh, ibool, is_acoustic):
    """Global points zeroed by enforce_acoustic_free_surface
    (enforce_acoustic_free_surface.f90:35-96): every GLL point of the listed
    free-surface edges of fluid elements, those of an external mesh
    (mesh.free_edges) or the structured mesh's outer edges
    (structured_free_edges)."""
    rows = mesh.free_edges if mesh.free_edges is not None else structured_free_edges(mesh, is_acoustic)
    pts = [int(ibool[e, j, i]) for (e, i0, i1, j0, j1) in rows if is_acoustic[e]
           for j in range(j0, j1 + 1) for i in range(i0, i1 + 1)]
    return np.unique(np.array(pts, dtype=np.int32)) if pts else np.zeros(0, np.int32)
