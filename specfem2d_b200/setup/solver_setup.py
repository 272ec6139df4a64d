"""Solver setup for the elastic time-marching path: produces the arrays the
C-ABI ``prepare_*`` entry points take.

Restated reference routines (0-based indices here):

* material stores -- src/specfem2D/setup_mesh.F90:524-800 and
  src/specfem2D/read_materials.f90:116-147 (kappa = lambda + mu in 2-D)
* mass matrix -- src/specfem2D/invert_mass_matrix.F90:34-466 (elastic,
  non-PML branch), the Newmark Stacey term :470-797, inversion :798-849
* Stacey edge normals/weights -- src/specfem2D/compute_stacey_elastic.f90:
  118-980 (left/right use the gamma-direction edge vector, bottom/top the
  xi-direction one; bottom/top skip points shared with a left/right edge)
* source location -- src/specfem2D/locate_source.F90:34-330; receivers --
  src/specfem2D/locate_receivers.F90:38-420 (nearest GLL point, then the
  elements touching its element's corners, NUM_ITER=5 Newton steps clamped
  to +-1.01)
* source arrays -- src/specfem2D/setup_sources_receivers.F90:925-1075 and
  src/specfem2D/compute_arrays_source.f90:34-110 (moment tensor)
* source time functions -- src/specfem2D/prepare_source_time_function.f90:
  160-260, src/specfem2D/comp_source_time_function.f90, t0 from
  src/specfem2D/set_source_parameters.f90:112-240
* receiver interpolation -- src/specfem2D/setup_sources_receivers.F90:1077-1138
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from .gll import GLL, NGLL, lagrange_any
from .mesh import (IBOTTOM, ILEFT, IRIGHT, ITOP, Mesh, createnum_fast, get_global,
                   recompute_jacobian, setup_mesh_coordinates)

PI = 3.141592653589793
HUGEVAL = 1.0e30
NUM_ITER = 5
f32 = np.float32

# LDDRK coefficients (6 stages), setup/constants.h.in:402-412 (CUSTOM_REAL)
ALPHA_LDDRK = np.array([0.0, -0.737101392796, -1.634740794341, -0.744739003780,
                        -1.469897351522, -2.813971388035], dtype=f32)
BETA_LDDRK = np.array([0.032918605146, 0.823256998200, 0.381530948900, 0.200092213184,
                       1.718581042715, 0.27], dtype=f32)
C_LDDRK = np.array([0.0, 0.032918605146, 0.249351723343, 0.466911705055, 0.582030414044,
                    0.847252983783], dtype=f32)


@dataclasses.dataclass
class Source:
    x: float
    z: float
    source_type: int = 1          # 1 = force, 2 = moment tensor
    time_function_type: int = 1   # 1 = Ricker, 2 = first derivative of Gaussian, 3 = Gaussian
    f0: float = 10.0
    tshift: float = 0.0
    anglesource_deg: float = 0.0
    Mxx: float = 1.0
    Mzz: float = 1.0
    Mxz: float = 0.0
    factor: float = 1.0


@dataclasses.dataclass
class Database:
    """Everything the time loop needs, in solver layout (see module docstring)."""

    nspec: int
    nglob: int
    ibool: np.ndarray
    xix: np.ndarray
    xiz: np.ndarray
    gammax: np.ndarray
    gammaz: np.ndarray
    jacobian: np.ndarray
    coord: np.ndarray
    rhostore: np.ndarray
    kappastore: np.ndarray
    mustore: np.ndarray
    rho_vpstore: np.ndarray
    rho_vsstore: np.ndarray
    rmass_inverse_elastic: np.ndarray   # (nglob, 2) f32
    # Stacey, one entry per absorbing GLL point in reference order
    stacey_iglob: np.ndarray            # (nabs_pts,) int32
    stacey_nx: np.ndarray               # f32
    stacey_nz: np.ndarray
    stacey_weight: np.ndarray           # jacobian1D * w
    stacey_rho_vp: np.ndarray
    stacey_rho_vs: np.ndarray
    # sources
    source_ispec: np.ndarray            # (nsrc,)
    sourcearrays: np.ndarray            # (nsrc, 5[j], 5[i], 2) f32
    stf: np.ndarray                     # (nsrc, nstep, nstage) f32
    # receivers
    rec_ispec: np.ndarray               # (nrec,)
    rec_xi: np.ndarray
    rec_gamma: np.ndarray
    hxir: np.ndarray                    # (nrec, 5) f64
    hgammar: np.ndarray
    rec_x: np.ndarray                   # final located x, z
    rec_z: np.ndarray
    cosrot: float
    sinrot: float
    # time
    nstep: int
    dt: float
    t0: float
    time_scheme: int                    # 1 Newmark, 2 LDDRK
    gll: GLL
    mesh: Mesh = None
    src_xi: np.ndarray = None
    src_gamma: np.ndarray = None
    # viscoelastic 3-SLS coefficients per GLL point and SLS (None = elastic):
    # keys a1, b1, a2, b2 (Newmark), itau1, phi1, itau2, phi2 (LDDRK), each (nspec, 5, 5, 3) f32
    atten: dict = None
    # anisotropy (None = isotropic): keys ispec (nspec,) bool, c11 c13 c15 c33 c35 c55 (nspec,5,5) f32
    aniso: dict = None
    # acoustic domain (None = no fluid element): keys ispec (nspec,) bool, rmass (nglob,) f32,
    # st_iglob/st_w/st_rvp (acoustic absorbing points), free_iglob (free-surface points),
    # cpl_ac_* and cpl_el_* (iglob, nx, nz, w per coupling point, acoustic and elastic side),
    # use_trick (USE_TRICK_FOR_BETTER_PRESSURE)
    acoustic: dict = None
    seismotype: int = 1                 # 1 displacement, 2 velocity, 3 acceleration, 4 pressure
    # CPML layers (None = none): keys region (nspec,) int (0 outside, 1 X, 2 Z, 3 XZ),
    # K_x K_z d_x d_z alpha_x alpha_z (nspec,5,5) float64, bnd_ac/bnd_el outer-edge points, dt
    pml: dict = None
    # analytical initial wavefield (None = start from rest): pot, pot_dot, pot_dot_dot (nglob,) f32
    # for a fluid, or displ, veloc, accel (nglob, 2) f32 for a solid
    initial_field: dict = None

    @property
    def deltat(self):
        return f32(self.dt)

    @property
    def deltatover2(self):
        return f32(0.5 * float(f32(self.dt)))

    @property
    def deltatsquareover2(self):
        d = float(f32(self.dt))
        return f32(0.5 * d * d)

    def element_order_colour(self):
        return None


def material_stores_from_velocity(rho, vp, vs, external: bool):
    """rhostore, kappastore, mustore, rho_vpstore, rho_vsstore (setup_mesh.F90:668-785).

    ``external`` follows the assign_external_model branch (vp, vs, rho given
    as CUSTOM_REAL per GLL point); otherwise the material-table branch
    (read_materials.f90:137-146: mu = rho cs^2, lambda = rho cp^2 - 2 mu,
    kappa = lambda + mu, vp recomputed from kappa and mu).
    """
    rho = np.asarray(rho, dtype=np.float64)
    vp = np.asarray(vp, dtype=np.float64)
    vs = np.asarray(vs, dtype=np.float64)
    if external:
        rhol = rho.astype(f32).astype(np.float64)
        vpl = vp.astype(f32).astype(np.float64)
        vsl = vs.astype(f32).astype(np.float64)
        mul = rhol * vsl * vsl
        kappal = rhol * vpl * vpl - mul
        vpu = vpl
    else:
        rhol = rho
        lambdaplus2mu = rho * vp * vp
        mul = rho * vs * vs
        lam = lambdaplus2mu - 2.0 * mul
        kappal = lam + mul
        vpu = np.sqrt((kappal + mul) / rhol)
    vsu = np.sqrt(mul / rhol)
    return dict(rhostore=rhol.astype(f32), kappastore=kappal.astype(f32), mustore=mul.astype(f32),
                rho_vpstore=(rhol * vpu).astype(f32), rho_vsstore=(rhol * vsu).astype(f32))


def _sequential_f32_accumulate(n, idx, contrib64, init=None):
    """acc[idx[k]] = f32(f64(acc[idx[k]]) + contrib64[k]) applied in k order."""
    acc = np.zeros(n, dtype=f32) if init is None else init.copy()
    order = np.argsort(idx, kind="stable")
    sidx = idx[order]
    start = np.r_[0, np.flatnonzero(np.diff(sidx)) + 1]
    counts = np.diff(np.r_[start, sidx.size])
    rank = np.arange(sidx.size) - np.repeat(start, counts)
    for r in range(int(rank.max()) + 1 if rank.size else 0):
        sel = order[rank == r]
        p = idx[sel]
        acc[p] = (acc[p].astype(np.float64) + contrib64[sel]).astype(f32)
    return acc


def _edge_points(mesh: Mesh, abs_corner_skip=True):
    """Yield (face k, type, list of (i, j)) for absorbing edges in reference order."""
    for k in range(len(mesh.abs_ispec)):
        t = int(mesh.abs_type[k])
        if t == ILEFT:
            pts = [(0, j) for j in range(NGLL)]
        elif t == IRIGHT:
            pts = [(NGLL - 1, j) for j in range(NGLL)]
        elif t == IBOTTOM:
            pts = [(i, 0) for i in range(NGLL)
                   if not (abs_corner_skip and ((mesh.abs_corner[k, 0] and i == 0)
                                                or (mesh.abs_corner[k, 1] and i == NGLL - 1)))]
        else:
            pts = [(i, NGLL - 1) for i in range(NGLL)
                   if not (abs_corner_skip and ((mesh.abs_corner[k, 2] and i == 0)
                                                or (mesh.abs_corner[k, 3] and i == NGLL - 1)))]
        yield k, t, pts


def edge_normal(geo: dict, gll: GLL, e: int, i: int, j: int, t: int):
    """Outward normal (nx, nz) and weight jacobian1D * w of GLL point (i, j) of
    element e on an edge of type t, in FP32 arithmetic
    (compute_stacey_elastic.f90:118-980, prepare_timerun.F90:1315-1430)."""
    jac = geo["jacobian"][e, j, i]
    if t in (ILEFT, IRIGHT):
        xgamma = f32(-geo["xiz"][e, j, i] * jac)
        zgamma = f32(geo["xix"][e, j, i] * jac)
        j1d = f32(np.sqrt(f32(f32(xgamma * xgamma) + f32(zgamma * zgamma))))
        if t == ILEFT:
            nx, nz = f32(-zgamma / j1d), f32(xgamma / j1d)
        else:
            nx, nz = f32(zgamma / j1d), f32(-xgamma / j1d)
        return nx, nz, f32(j1d * gll.wzgll[j])
    xxi = f32(geo["gammaz"][e, j, i] * jac)
    zxi = f32(-geo["gammax"][e, j, i] * jac)
    j1d = f32(np.sqrt(f32(f32(xxi * xxi) + f32(zxi * zxi))))
    if t == IBOTTOM:
        nx, nz = f32(zxi / j1d), f32(-xxi / j1d)
    else:
        nx, nz = f32(-zxi / j1d), f32(xxi / j1d)
    return nx, nz, f32(j1d * gll.wxgll[i])


def stacey_points(mesh: Mesh, geo: dict, mat: dict, ibool, gll: GLL, stacey: bool, elastic=None):
    """Per absorbing GLL point of an elastic element (all elements when
    ``elastic`` is None): iglob, normal, weight, rho*vp, rho*vs in FP32 arithmetic."""
    out = {k: [] for k in ("iglob", "nx", "nz", "w", "rvp", "rvs")}
    if stacey and mesh.abs_ispec is not None:
        for k, t, pts in _edge_points(mesh):
            e = int(mesh.abs_ispec[k])
            if elastic is not None and not elastic[e]:
                continue
            for (i, j) in pts:
                nx, nz, w = edge_normal(geo, gll, e, i, j, t)
                out["iglob"].append(int(ibool[e, j, i]))
                out["nx"].append(nx)
                out["nz"].append(nz)
                out["w"].append(w)
                out["rvp"].append(mat["rho_vpstore"][e, j, i])
                out["rvs"].append(mat["rho_vsstore"][e, j, i])
    return (np.array(out["iglob"], dtype=np.int32), np.array(out["nx"], dtype=f32),
            np.array(out["nz"], dtype=f32), np.array(out["w"], dtype=f32),
            np.array(out["rvp"], dtype=f32), np.array(out["rvs"], dtype=f32))


def mass_matrix_elastic(ibool, nglob, geo, mat, gll: GLL, stacey_pts, newmark: bool, dt: float, elastic=None,
                        pml=None):
    """rmass_inverse_elastic (nglob, 2) f32 (invert_mass_matrix.F90:34-849, elastic).

    Only elastic elements contribute (all when ``elastic`` is None); points
    with no elastic mass get 1 before inversion (invert_mass_matrix.F90:820-822).
    PML elements (``pml`` dict of setup.pml) carry their K and d dt/2 factors."""
    wxwz = (gll.wxgll[None, :] * gll.wzgll[:, None]).astype(f32)  # [j][i], CUSTOM_REAL product
    el = np.arange(ibool.shape[0]) if elastic is None else np.flatnonzero(elastic)
    contrib = (wxwz[None].astype(np.float64) * mat["rhostore"][el].astype(np.float64)
               * geo["jacobian"][el].astype(np.float64))
    if pml is not None:
        from .pml import mass_entries

        base = ((wxwz[None] * mat["rhostore"][el].astype(f32)).astype(f32) * geo["jacobian"][el].astype(f32)).astype(f32)
        base = base[pml["region"][el] > 0]
        idx, val = mass_entries(ibool, el, contrib, base, pml, newmark, float(f32(0.5 * float(f32(dt)))))
        m = _sequential_f32_accumulate(nglob, idx, val)
    else:
        m = _sequential_f32_accumulate(nglob, ibool[el].ravel(), contrib.ravel())
    mx = m.copy()
    mz = m.copy()
    if newmark and len(stacey_pts[0]):
        iglob, nxs, nzs, ws, rvp, rvs = stacey_pts
        dto2 = f32(0.5 * float(f32(dt)))
        for p in range(len(iglob)):
            vx = dto2
            vz = dto2
            nx, nz = nxs[p], nzs[p]
            vn = f32(f32(nx * vx) + f32(nz * vz))
            tx = f32(f32(f32(rvp[p] * vn) * nx) + f32(rvs[p] * f32(vx - f32(vn * nx))))
            tz = f32(f32(f32(rvp[p] * vn) * nz) + f32(rvs[p] * f32(vz - f32(vn * nz))))
            g = iglob[p]
            mx[g] = f32(mx[g] + f32(tx * ws[p]))
            mz[g] = f32(mz[g] + f32(tz * ws[p]))
    mx = np.where(mx <= 0, f32(1.0), mx).astype(f32)
    mz = np.where(mz <= 0, f32(1.0), mz).astype(f32)
    return np.stack([f32(1.0) / mx, f32(1.0) / mz], axis=1).astype(f32)


class _PointLocator:
    """Nearest-GLL-point search with the reference's tie rule.

    The reference scans (ispec, j, i) in order and keeps the first strict
    minimum of the squared distance (locate_receivers.F90:150-170).  A k-d
    tree finds the nearest global points; among the element-local
    occurrences of all points at that exact distance the first in scan order
    wins, which is the same answer.
    """

    def __init__(self, ibool, coord):
        from scipy.spatial import cKDTree

        self.ibool = ibool
        self.coord = coord
        self.tree = cKDTree(coord)
        flat = ibool.ravel()
        first = np.full(coord.shape[0], flat.size, dtype=np.int64)
        # first occurrence of every point in scan order: with a repeated index the
        # last assignment wins, so the occurrences are written in reverse order
        first[flat[::-1]] = np.arange(flat.size - 1, -1, -1, dtype=np.int64)
        self.first = first
        # corner point -> elements having it as a corner (CSR), for the candidate search
        corners = ibool[:, [0, 0, NGLL - 1, NGLL - 1], [0, NGLL - 1, 0, NGLL - 1]].ravel()
        order = np.argsort(corners, kind="stable")
        self.corner_elems = (order // 4).astype(np.int64)
        self.corner_ptr = np.searchsorted(corners[order], np.arange(coord.shape[0] + 1))

    def elements_touching(self, points):
        """Ascending element ids that have any of `points` as a corner."""
        parts = [self.corner_elems[self.corner_ptr[g]:self.corner_ptr[g + 1]] for g in points]
        return np.unique(np.concatenate(parts)) if parts else np.zeros(0, dtype=np.int64)

    def nearest_flat(self, x_t, z_t):
        k = min(16, self.coord.shape[0])
        _, idx = self.tree.query([x_t, z_t], k=k)
        idx = np.atleast_1d(idx)
        d2 = (x_t - self.coord[idx, 0]) ** 2 + (z_t - self.coord[idx, 1]) ** 2
        best = idx[d2 == d2.min()]
        return int(self.first[best].min())


def _locate(mesh: Mesh, ibool, coord, gll: GLL, x_t: float, z_t: float, iterate: bool = True, locator=None):
    """Shared body of locate_source / locate_receivers: returns (ispec, xi, gamma, x, z)."""
    if locator is None:
        locator = _PointLocator(ibool, coord)
    k = locator.nearest_flat(x_t, z_t)
    ispec0 = k // (NGLL * NGLL)
    ix0 = k % NGLL
    iz0 = (k // NGLL) % NGLL
    corners = {int(ibool[ispec0, 0, 0]), int(ibool[ispec0, 0, NGLL - 1]),
               int(ibool[ispec0, NGLL - 1, NGLL - 1]), int(ibool[ispec0, NGLL - 1, 0])}
    cand = [ispec0]
    for e in locator.elements_touching(sorted(corners)):
        if int(e) != ispec0:
            cand.append(int(e))
    best = (HUGEVAL, None)
    for n, e in enumerate(cand):
        if n > 0:
            ix0 = int(NGLL / 2.0) - 1  # Fortran int(NGLLX/2.0) = 2, 1-based
            iz0 = int(NGLL / 2.0) - 1
        xi = float(gll.xigll[ix0])
        gamma = float(gll.zigll[iz0])
        if iterate:
            for _ in range(NUM_ITER):
                x, z, xix, xiz, gammax, gammaz, _ = recompute_jacobian(mesh, e, xi, gamma)
                dx = -(x - x_t)
                dz = -(z - z_t)
                dxi = xix * dx + xiz * dz
                dgamma = gammax * dx + gammaz * dz
                xi = xi + dxi
                gamma = gamma + dgamma
                xi = min(max(xi, -1.01), 1.01)
                gamma = min(max(gamma, -1.01), 1.01)
        x, z, *_ = recompute_jacobian(mesh, e, xi, gamma)
        dist = math.sqrt((x_t - x) ** 2 + (z_t - z) ** 2)
        if dist < best[0]:
            best = (dist, (e, xi, gamma, x, z))
    return best[1]


def source_time_function(src: Source, t0: float, dt: float, nstep: int, time_scheme: int,
                         use_trick: bool = False):
    """(nstep, nstage) f32 values of -factor * stf(t) (prepare_source_time_function.f90).

    ``use_trick`` (USE_TRICK_FOR_BETTER_PRESSURE) replaces each time function
    by its second derivative (the Ricker by the fourth derivative of the
    Gaussian, the first derivative by the third, the Gaussian by the second;
    prepare_source_time_function.f90:205-262, comp_source_time_function.f90:90-143),
    so that -chi rather than -chi_dd is the pressure."""
    if use_trick and src.time_function_type not in (1, 2, 3):
        raise NotImplementedError("USE_TRICK_FOR_BETTER_PRESSURE is restated for the Ricker and Gaussian families")
    nstage = 1 if time_scheme == 1 else 6
    out = np.zeros((nstep, nstage), dtype=f32)
    a = PI ** 2 * src.f0 ** 2
    for it in range(1, nstep + 1):
        for s in range(nstage):
            if time_scheme == 1:
                timeval = float(it - 1) * dt
            else:
                timeval = float(it - 1 - 1) * dt + float(C_LDDRK[s]) * dt
            t = timeval - t0 - src.tshift
            if src.time_function_type == 1 and use_trick:
                v = -2.0 * a * (3.0 - 12.0 * a * t * t + 4.0 * a ** 2 * t * t * t * t) * math.exp(-a * t * t)
            elif src.time_function_type == 1 or (src.time_function_type == 3 and use_trick):
                # Ricker; with the trick also the second derivative of the Gaussian (case 3)
                v = (1.0 - 2.0 * a * t ** 2) * math.exp(-a * t ** 2)
            elif src.time_function_type == 2 and use_trick:
                v = 2.0 * a * t * math.exp(-a * t ** 2) * (-3.0 + 2.0 * a * t ** 2)
            elif src.time_function_type == 2:
                v = t * math.exp(-a * t ** 2)
            elif src.time_function_type == 3:
                v = -math.exp(-a * t ** 2) / (2.0 * a)
            else:
                raise NotImplementedError("time_function_type")
            out[it - 1, s] = f32(-src.factor * v)
    return out


def compute_t0(sources, user_t0: float = 0.0):
    """Simulation start time (set_source_parameters.f90:112-240), Ricker/Gaussian family."""
    t0s = [1.20 * (1.0 / s.f0) + s.tshift for s in sources]
    if len(sources) == 1:
        t0 = t0s[0]
        min_tshift = sources[0].tshift
        sources[0].tshift = 0.0
    else:
        t0 = min(t0s)
        min_tshift = min(s.tshift for s in sources)
        for s, t in zip(sources, t0s):
            s.tshift = t - t0
    if t0 <= user_t0 + min_tshift:
        t0 = user_t0
        for s, t in zip(sources, t0s):
            s.tshift = t - 1.20 * (1.0 / s.f0)
    return t0


def build_database(mesh: Mesh, rho, vp, vs, sources, receivers_xz, nstep: int, dt: float,
                   stacey: bool = True, external_model: bool = True, time_scheme: int = 1,
                   user_t0: float = 0.0, anglerec_deg: float = 0.0, qkappa=None, qmu=None,
                   attenuation_f0: float | None = None, use_trick: bool = False,
                   seismotype: int = 1, pml: dict | None = None, initialfield: bool = False) -> Database:
    """Run the host setup chain and return a Database.

    ``rho, vp, vs`` are per-GLL-point arrays (nspec,5,5) (external model) or
    scalars/arrays used through the material-table branch when
    ``external_model`` is False.  Elements with vs = 0 are acoustic (fluid);
    the acoustic domain, its absorbing points, free surface and the
    fluid-solid coupling go into ``Database.acoustic``.  ``seismotype`` 4
    records pressure (receivers in acoustic elements).  ``pml`` (keys
    nelem_thickness, and optionally k_min, k_max, damping_acoustic,
    damping_elastic) puts CPML layers on the absorbing sides instead of
    Stacey conditions; the profiles go into ``Database.pml``.  With
    ``initialfield`` the sources set t0 only: none is injected, and the
    analytical initial wavefield of the first source's type goes into
    ``Database.initial_field`` (prepare_initial_field.F90).
    """
    from . import acoustic as ac_setup

    gll = GLL()
    ib0, nglob = createnum_fast(mesh, gll)
    ibool = get_global(ib0)
    geo = setup_mesh_coordinates(mesh, gll, ibool, nglob)
    shp = (mesh.nspec, NGLL, NGLL)
    rho = np.broadcast_to(np.asarray(rho, dtype=np.float64), shp)
    vp = np.broadcast_to(np.asarray(vp, dtype=np.float64), shp)
    vs = np.broadcast_to(np.asarray(vs, dtype=np.float64), shp)
    mat = material_stores_from_velocity(rho, vp, vs, external_model)
    is_ac = ac_setup.acoustic_element_flags(vs)
    elastic = None if not is_ac.any() else ~is_ac
    pml_db = None
    if pml is not None:
        from . import pml as pml_setup

        if stacey:
            raise ValueError("CPML and Stacey conditions are exclusive")
        is_pml, region, _ = pml_setup.pml_elements(mesh, ibool, int(pml["nelem_thickness"]))
        coefs = pml_setup.pml_coefficients(
            ibool, geo["coord"], is_pml, region, mat["rho_vpstore"], mat["rhostore"], is_ac,
            max(s_.f0 for s_ in sources), pml.get("k_min", 1.0), pml.get("k_max", 1.0),
            pml.get("damping_acoustic", 0.5), pml.get("damping_elastic", 1.0))
        bnd_ac, bnd_el = pml_setup.pml_boundary_points(mesh, ibool, is_pml, is_ac)
        pml_db = dict(region=region, bnd_ac=bnd_ac, bnd_el=bnd_el, dt=float(dt), **coefs)
    spts = stacey_points(mesh, geo, mat, ibool, gll, stacey, elastic)
    rmass = mass_matrix_elastic(ibool, nglob, geo, mat, gll, spts, time_scheme == 1, dt, elastic, pml_db)
    acoustic = None
    if is_ac.any():
        edges = ac_setup.coupling_edges(ibool, is_ac)
        cpl_ac, cpl_el = ac_setup.coupling_points(edges, ibool, geo, gll)
        if stacey:
            st_ac = ac_setup.stacey_acoustic_points(mesh, geo, mat, ibool, gll, is_ac, edges)
        else:
            st_ac = (np.zeros(0, np.int32), np.zeros(0, f32), np.zeros(0, f32))
        acoustic = dict(
            ispec=is_ac,
            rmass=ac_setup.mass_matrix_acoustic(ibool, nglob, geo, mat, gll, is_ac, st_ac, time_scheme == 1, dt,
                                                pml_db),
            st_iglob=st_ac[0], st_w=st_ac[1], st_rvp=st_ac[2],
            free_iglob=ac_setup.free_surface_points(mesh, ibool, is_ac),
            cpl_ac_iglob=cpl_ac[0], cpl_ac_nx=cpl_ac[1], cpl_ac_nz=cpl_ac[2], cpl_ac_w=cpl_ac[3],
            cpl_el_iglob=cpl_el[0], cpl_el_nx=cpl_el[1], cpl_el_nz=cpl_el[2], cpl_el_w=cpl_el[3],
            cpl_ac_elpt=cpl_ac[4], cpl_el_acpt=cpl_el[4],
            use_trick=bool(use_trick))
    coord = geo["coord"]
    t0 = compute_t0(sources, user_t0)
    nstage = 1 if time_scheme == 1 else 6
    src_ispec, src_arr, src_stf, sxi, sgam = [], [], [], [], []
    locator = _PointLocator(ibool, coord)
    init = None
    if initialfield:
        # setup_sources_receivers.F90:958-961: no source arrays with an initial field
        from .initial_field import initial_mode_field

        if not sources or sources[0].source_type != 6:
            raise NotImplementedError("initial fields: only the membrane mode (source_type 6) is restated")
        init = initial_mode_field(coord, mat["rho_vpstore"], mat["rhostore"], t0, acoustic=bool(is_ac.any()))
    for s in ([] if initialfield else sources):
        e, xi, gamma, _, _ = _locate(mesh, ibool, coord, gll, s.x, s.z, iterate=True, locator=locator)
        hx, hpx = lagrange_any(xi, gll.xigll)
        hg, hpg = lagrange_any(gamma, gll.zigll)
        arr = np.zeros((NGLL, NGLL, 2), dtype=f32)
        if is_ac[e]:
            # pressure source: sourcearray = hlagrange (setup_sources_receivers.F90:1003-1006)
            if s.source_type != 1:
                raise ValueError("a moment-tensor source cannot sit in an acoustic element")
            for j in range(NGLL):
                for i in range(NGLL):
                    arr[j, i, :] = f32(hx[i] * hg[j])
        elif s.source_type == 1:
            ang = s.anglesource_deg * PI / 180.0
            for j in range(NGLL):
                for i in range(NGLL):
                    h = hx[i] * hg[j]
                    arr[j, i, 0] = f32(math.sin(ang) * h)
                    arr[j, i, 1] = f32(-math.cos(ang) * h)
        else:
            dxis_dx = dxis_dz = dgam_dx = dgam_dz = 0.0
            for m in range(NGLL):
                for k in range(NGLL):
                    h = hx[k] * hg[m]
                    dxis_dx = dxis_dx + h * float(geo["xix"][e, m, k])
                    dxis_dz = dxis_dz + h * float(geo["xiz"][e, m, k])
                    dgam_dx = dgam_dx + h * float(geo["gammax"][e, m, k])
                    dgam_dz = dgam_dz + h * float(geo["gammaz"][e, m, k])
            for m in range(NGLL):
                for k in range(NGLL):
                    dsx = (hpx[k] * dxis_dx) * hg[m] + hx[k] * (hpg[m] * dgam_dx)
                    dsz = (hpx[k] * dxis_dz) * hg[m] + hx[k] * (hpg[m] * dgam_dz)
                    arr[m, k, 0] = f32(s.Mxx * dsx + s.Mxz * dsz)
                    arr[m, k, 1] = f32(s.Mxz * dsx + s.Mzz * dsz)
        src_ispec.append(e)
        src_arr.append(arr)
        src_stf.append(source_time_function(s, t0, dt, nstep, time_scheme, use_trick))
        sxi.append(xi)
        sgam.append(gamma)
    rec_ispec, rxi, rgam, hxr, hgr, rxx, rzz = [], [], [], [], [], [], []
    for (xr, zr) in receivers_xz:
        e, xi, gamma, x, z = _locate(mesh, ibool, coord, gll, xr, zr, iterate=True, locator=locator)
        hx, _ = lagrange_any(xi, gll.xigll)
        hg, _ = lagrange_any(gamma, gll.zigll)
        rec_ispec.append(e); rxi.append(xi); rgam.append(gamma)
        hxr.append(hx); hgr.append(hg); rxx.append(x); rzz.append(z)
    ang = anglerec_deg * PI / 180.0
    atten = None
    if qkappa is not None and qmu is not None:
        from .attenuation import attenuation_arrays

        f0_ref = attenuation_f0
        if sources and sources[0].time_function_type not in (4, 5):
            f0_ref = sources[0].f0  # prepare_attenuation.f90:319-321
        qk_all = np.broadcast_to(np.asarray(qkappa, dtype=np.float64), shp)
        qm_all = np.broadcast_to(np.asarray(qmu, dtype=np.float64), shp)
        atten = attenuation_arrays(qk_all, qm_all, f0_ref, dt)
        if pml_db is not None:
            # layer elements whose largest Qkappa and Qmu are both below 9998.999 take the
            # viscoelastic CPML update, the others the elastic one
            # (compute_forces_viscoelastic.F90:178-181, 249-267)
            low = (qk_all.reshape(mesh.nspec, -1).max(axis=1) < 9998.999) & \
                  (qm_all.reshape(mesh.nspec, -1).max(axis=1) < 9998.999)
            pml_db["visco"] = ((np.asarray(pml_db["region"]) > 0) & low & ~is_ac).astype(np.int32)
    return Database(
        nspec=mesh.nspec, nglob=nglob, ibool=ibool.astype(np.int32),
        xix=geo["xix"], xiz=geo["xiz"], gammax=geo["gammax"], gammaz=geo["gammaz"],
        jacobian=geo["jacobian"], coord=coord, **mat,
        rmass_inverse_elastic=rmass,
        stacey_iglob=spts[0], stacey_nx=spts[1], stacey_nz=spts[2], stacey_weight=spts[3],
        stacey_rho_vp=spts[4], stacey_rho_vs=spts[5],
        source_ispec=np.array(src_ispec, dtype=np.int32),
        sourcearrays=np.array(src_arr, dtype=f32).reshape(len(src_ispec), NGLL, NGLL, 2),
        stf=np.array(src_stf, dtype=f32).reshape(len(src_ispec), nstep, nstage),
        rec_ispec=np.array(rec_ispec, dtype=np.int32), rec_xi=np.array(rxi), rec_gamma=np.array(rgam),
        hxir=np.array(hxr).reshape(-1, NGLL), hgammar=np.array(hgr).reshape(-1, NGLL),
        rec_x=np.array(rxx), rec_z=np.array(rzz),
        cosrot=math.cos(ang), sinrot=math.sin(ang),
        nstep=nstep, dt=dt, t0=t0, time_scheme=time_scheme, gll=gll, mesh=mesh,
        src_xi=np.array(sxi), src_gamma=np.array(sgam), atten=atten, acoustic=acoustic,
        seismotype=int(seismotype), pml=pml_db, initial_field=init)
