"""Python host binding of libsf2d_b200.so (the sm_100a C ABI in include/sf2d_b200.h).

This is the product's host side: it turns a setup Database into the
reference-layout descriptor the C ABI takes and drives the device time loop.
There is no CPU fallback: if the CUDA library is missing or fails, calls raise.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .build import LIB

_f = ctypes.POINTER(ctypes.c_float)
_d = ctypes.POINTER(ctypes.c_double)
_i = ctypes.POINTER(ctypes.c_int)

SF2D_OK = 0
SF2D_ERR_INVALID = -1
SF2D_ERR_CUDA = -2
SF2D_ERR_OOM = -3
SF2D_ERR_UNSTABLE = -4
SF2D_ERR_TIMEOUT = -5


class SF2DError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"sf2d error {code}: {msg}")
        self.code = code


class UnstableError(SF2DError):
    pass


class SolverTimeout(SF2DError):
    """synchronize() gave up waiting; the queued steps keep running."""


class ElasticDesc(ctypes.Structure):
    _fields_ = [
        ("nspec", ctypes.c_int), ("nglob", ctypes.c_int),
        ("ibool", _i),
        ("xix", _f), ("xiz", _f), ("gammax", _f), ("gammaz", _f),
        ("lambdastore", _f), ("mustore", _f),
        ("rmass_inverse", _f),
        ("hprime", _f), ("hprimewgll", _f), ("wxgll", _f), ("wzgll", _f),
        ("centroid_xz", _d),
        ("nstacey", ctypes.c_int), ("st_iglob", _i),
        ("st_nx", _f), ("st_nz", _f), ("st_w", _f), ("st_rho_vp", _f), ("st_rho_vs", _f),
        ("nsrc", ctypes.c_int), ("src_ispec", _i), ("sourcearrays", _f), ("stf", _f),
        ("nrec", ctypes.c_int), ("rec_ispec", _i), ("hxir", _d), ("hgammar", _d),
        ("cosrot", ctypes.c_double), ("sinrot", ctypes.c_double), ("seismotype", ctypes.c_int),
        ("nstep", ctypes.c_int),
        ("deltat", ctypes.c_float), ("deltatover2", ctypes.c_float), ("deltatsquareover2", ctypes.c_float),
        ("tile_elems", ctypes.c_int), ("threads_per_block", ctypes.c_int),
        ("time_scheme", ctypes.c_int), ("nstage", ctypes.c_int),
        ("alpha_lddrk", _f), ("beta_lddrk", _f),
        ("ispec_is_anisotropic", _i),
        ("c11", _f), ("c13", _f), ("c15", _f), ("c33", _f), ("c35", _f), ("c55", _f),
        ("att_a1", _f), ("att_b1", _f), ("att_a2", _f), ("att_b2", _f),
        ("att_itau1", _f), ("att_phi1", _f), ("att_itau2", _f), ("att_phi2", _f),
        ("pml_region", _i),
        ("pml_K_x", _d), ("pml_K_z", _d), ("pml_d_x", _d), ("pml_d_z", _d), ("pml_alpha_x", _d), ("pml_alpha_z", _d),
        ("rhostore", _f), ("jacobian", _f),
        ("npml_edge", ctypes.c_int), ("pml_edge_iglob", _i),
        ("pml_dt", ctypes.c_double),
        ("pml_visco", _i), ("att_teps1", _f), ("att_teps2", _f), ("att_mu1", _f), ("att_mu2", _f),
        ("pml_tile_elems", ctypes.c_int), ("pml_threads_per_block", ctypes.c_int),
    ]


_lib = None


def load_library(path: str = LIB):
    """Load the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"CUDA extension not built: {path} (run python -m specfem2d_b200.build)")
    lib = ctypes.CDLL(path)
    vp = ctypes.c_void_p
    sigs = {
        "sf2d_initialize_device": [ctypes.c_int, ctypes.POINTER(ctypes.c_int)],
        "sf2d_elastic_create": [ctypes.POINTER(ElasticDesc), ctypes.POINTER(vp)],
        "sf2d_set_fields": [vp, _f, _f, _f],
        "sf2d_get_fields": [vp, _f, _f, _f],
        "sf2d_run": [vp, ctypes.c_int, _d],
        "sf2d_enqueue": [vp, ctypes.c_int],
        "sf2d_prepare": [vp],
        "sf2d_synchronize": [vp, ctypes.c_double],
        "sf2d_copy_seismograms": [vp, ctypes.c_int, ctypes.c_int, _d],
        "sf2d_get_norm": [vp, _f],
        "sf2d_step_index": [vp, _i],
        "sf2d_get_stream": [vp, ctypes.POINTER(vp)],
        "sf2d_time_kernels": [vp, ctypes.c_int, _f],
        "sf2d_layout_info": [vp, ctypes.POINTER(ctypes.c_longlong)],
        "sf2d_launch_count": [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_longlong)],
        "sf2d_destroy": [vp],
        "sf2d_fwi_create": [ctypes.POINTER(ElasticDesc), _f, _f, ctypes.c_int, ctypes.POINTER(vp)],
        "sf2d_fwi_forward": [vp, _d],
        "sf2d_fwi_backward": [vp, _f, _f, _f, _f],
        "sf2d_fwi_adjoint_seismograms": [vp, _d],
        "sf2d_smooth": [ctypes.c_int, _f, _f, _f, _f, ctypes.c_int, _f, ctypes.c_float, ctypes.c_float,
                        ctypes.c_float, _f, vp],
        "sf2d_fwi_enable_hessian": [vp],
        "sf2d_fwi_hessian": [vp, _f, _f],
        "sf2d_set_members": [vp, _i, ctypes.c_int],
        "sf2d_member_status": [vp, _i],
        "sf2d_fwi_destroy": [vp],
        "sf2d_member_norms_noalloc": [vp, ctypes.POINTER(ctypes.c_int64), ctypes.c_int, _f, vp],
    }
    for name, args in sigs.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = ctypes.c_int
    lib.sf2d_tiling_stats.argtypes = [ctypes.c_int, ctypes.c_int, _i, _d, ctypes.c_int,
                                      ctypes.POINTER(ctypes.c_longlong)]
    lib.sf2d_tiling_stats.restype = ctypes.c_int
    lib.sf2d_last_error.restype = ctypes.c_char_p
    lib.sf2d_last_error.argtypes = []
    _lib = lib
    return lib


def _seis_buffer(nrec: int, nstep: int, out=None):
    if out is None:
        return np.zeros((nrec, nstep, 2), dtype=np.float64)
    if out.shape != (nrec, nstep, 2) or out.dtype != np.float64 or not out.flags.c_contiguous:
        raise ValueError(f"seismogram buffer must be C-contiguous float64 of shape {(nrec, nstep, 2)}")
    return out


def initialize_device(rank: int) -> int:
    """Make device rank % (visible devices) current for this thread in the
    library's own CUDA runtime (the reference's initialize_cuda_device); call it
    with the same number given to torch.cuda.set_device.  Returns the number of
    visible devices."""
    n = ctypes.c_int(0)
    _check(load_library().sf2d_initialize_device(int(rank), ctypes.byref(n)))
    return int(n.value)


def _check(rc):
    if rc == SF2D_OK:
        return
    msg = load_library().sf2d_last_error().decode(errors="replace")
    if rc == SF2D_ERR_UNSTABLE:
        raise UnstableError(rc, msg)
    if rc == SF2D_ERR_TIMEOUT:
        raise SolverTimeout(rc, msg)
    raise SF2DError(rc, msg)


def lambda_store(db) -> np.ndarray:
    """lambda per GLL point formed in FP32 exactly as the CPU solver does:
    cpl = rho_vp / rho, lambda = rho*cpl*cpl - 2*mu (compute_forces_viscoelastic.F90:286-294)."""
    f32 = np.float32
    rho = db.rhostore.astype(f32)
    cpl = (db.rho_vpstore.astype(f32) / rho).astype(f32)
    return ((rho * cpl).astype(f32) * cpl - f32(2.0) * db.mustore.astype(f32)).astype(f32)


def element_centroids(db) -> np.ndarray:
    """Element centres (mean of the four corner GLL points) used to order tiles."""
    ib = db.ibool
    c = db.coord[ib[:, [0, 0, 4, 4], [0, 4, 0, 4]]]  # (nspec, 4, 2)
    return np.ascontiguousarray(c.mean(axis=1))


def tiling_stats(db, tile_elems: int = 64):
    """Host-only tiling check (no GPU): returns the statistics dict or raises."""
    lib = load_library()
    ib = np.ascontiguousarray(db.ibool, dtype=np.int32)
    cen = element_centroids(db)
    out = (ctypes.c_longlong * 8)()
    rc = lib.sf2d_tiling_stats(db.nspec, db.nglob, ib.ctypes.data_as(_i), cen.ctypes.data_as(_d),
                               tile_elems, out)
    if rc != 0:
        raise SF2DError(rc, "tiling invariant violated")
    keys = ["ntiles", "nshared", "max_local", "max_elems", "max_colours", "n_interior", "n_slots", "reserved"]
    return dict(zip(keys, [int(x) for x in out]))


def smooth(db, fields, sigma_h: float, sigma_v: float, cutoff: float = 6.0) -> np.ndarray:
    """Gaussian smoothing of per-element-point fields (nfields <= 4, each
    (nspec, 5, 5)) on the GPU, as smooth_sem.F90 smooths sensitivity kernels:
    horizontal and vertical standard deviations sigma_h, sigma_v in metres,
    points within `cutoff` standard deviations."""
    lib = load_library()
    fl = np.ascontiguousarray(np.asarray(fields, dtype=np.float32).reshape(-1, db.nspec, 5, 5))
    x = np.ascontiguousarray(db.coord[db.ibool, 0], dtype=np.float32)
    z = np.ascontiguousarray(db.coord[db.ibool, 1], dtype=np.float32)
    jac = np.ascontiguousarray(db.jacobian, dtype=np.float32)
    w = db.gll.wgll_dble
    wsq = np.ascontiguousarray((w[None, :] * w[:, None]).astype(np.float32))
    out = np.zeros_like(fl)
    _check(lib.sf2d_smooth(int(db.nspec), x.ctypes.data_as(_f), z.ctypes.data_as(_f), jac.ctypes.data_as(_f),
                           wsq.ctypes.data_as(_f), fl.shape[0], fl.ctypes.data_as(_f), float(sigma_h),
                           float(sigma_v), float(cutoff), out.ctypes.data_as(_f), None))
    return out


def member_norms_noalloc(field_ptr: int, offsets, stream: int = 0) -> np.ndarray:
    """Maximum displacement norm per batch member of a caller-owned device
    field of (ux, uz) float pairs at device address `field_ptr`; member m is
    points offsets[m]:offsets[m+1].  Allocates no device memory (the library
    keeps its intermediates in a static device array), for callers whose
    device memory is all owned by another allocator."""
    lib = load_library()
    off = np.ascontiguousarray(offsets, dtype=np.int64)
    out = np.zeros(max(len(off) - 1, 0), dtype=np.float32)
    _check(lib.sf2d_member_norms_noalloc(ctypes.c_void_p(field_ptr), off.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                         len(off) - 1, out.ctypes.data_as(_f), ctypes.c_void_p(stream)))
    return out


def build_desc(db, tile_elems: int = 32, seismotype: int = 1, threads_per_block: int = 256,
               pml_tile_elems: int = 0, pml_threads_per_block: int = 0):
    """sf2d_elastic_desc for a setup Database; returns (desc, arrays kept alive)."""
    keep = []

    def f(a):
        arr = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
        keep.append(arr)
        return arr.ctypes.data_as(_f)

    def dd(a):
        arr = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
        keep.append(arr)
        return arr.ctypes.data_as(_d)

    def i(a):
        arr = np.ascontiguousarray(np.asarray(a, dtype=np.int32))
        keep.append(arr)
        return arr.ctypes.data_as(_i)

    g = db.gll
    d = ElasticDesc()
    d.nspec, d.nglob = db.nspec, db.nglob
    d.ibool = i(db.ibool)
    d.xix, d.xiz, d.gammax, d.gammaz = f(db.xix), f(db.xiz), f(db.gammax), f(db.gammaz)
    d.lambdastore, d.mustore = f(lambda_store(db)), f(db.mustore)
    d.rmass_inverse = f(db.rmass_inverse_elastic)
    d.hprime, d.hprimewgll, d.wxgll, d.wzgll = f(g.hprime), f(g.hprimewgll), f(g.wxgll), f(g.wzgll)
    d.centroid_xz = dd(element_centroids(db))
    d.nstacey = len(db.stacey_iglob)
    d.st_iglob = i(db.stacey_iglob)
    d.st_nx, d.st_nz, d.st_w = f(db.stacey_nx), f(db.stacey_nz), f(db.stacey_weight)
    d.st_rho_vp, d.st_rho_vs = f(db.stacey_rho_vp), f(db.stacey_rho_vs)
    d.nsrc = len(db.source_ispec)
    d.src_ispec = i(db.source_ispec)
    d.sourcearrays = f(db.sourcearrays)
    d.stf = f(db.stf)
    d.nstage = int(db.stf.shape[2])
    d.nrec = len(db.rec_ispec)
    d.rec_ispec = i(db.rec_ispec)
    d.hxir, d.hgammar = dd(db.hxir), dd(db.hgammar)
    d.cosrot, d.sinrot = float(db.cosrot), float(db.sinrot)
    d.seismotype = seismotype
    d.nstep = db.nstep
    d.deltat, d.deltatover2, d.deltatsquareover2 = (float(db.deltat), float(db.deltatover2),
                                                    float(db.deltatsquareover2))
    d.tile_elems = tile_elems
    d.threads_per_block = threads_per_block
    d.pml_tile_elems, d.pml_threads_per_block = pml_tile_elems, pml_threads_per_block
    from .setup.solver_setup import ALPHA_LDDRK, BETA_LDDRK

    d.time_scheme = int(db.time_scheme)
    d.alpha_lddrk, d.beta_lddrk = f(ALPHA_LDDRK), f(BETA_LDDRK)
    an = getattr(db, "aniso", None)
    if an is not None:
        d.ispec_is_anisotropic = i(an["ispec"].astype(np.int32))
        d.c11, d.c13, d.c15 = f(an["c11"]), f(an["c13"]), f(an["c15"])
        d.c33, d.c35, d.c55 = f(an["c33"]), f(an["c35"]), f(an["c55"])
    at = getattr(db, "atten", None)
    if at is not None:
        if int(db.time_scheme) == 1:
            d.att_a1, d.att_b1, d.att_a2, d.att_b2 = f(at["a1"]), f(at["b1"]), f(at["a2"]), f(at["b2"])
        else:
            d.att_itau1, d.att_phi1 = f(at["itau1"]), f(at["phi1"])
            d.att_itau2, d.att_phi2 = f(at["itau2"]), f(at["phi2"])
    pm = getattr(db, "pml", None)
    if pm is not None:
        d.pml_region = i(pm["region"])
        d.pml_K_x, d.pml_K_z = dd(pm["K_x"]), dd(pm["K_z"])
        d.pml_d_x, d.pml_d_z = dd(pm["d_x"]), dd(pm["d_z"])
        d.pml_alpha_x, d.pml_alpha_z = dd(pm["alpha_x"]), dd(pm["alpha_z"])
        d.rhostore, d.jacobian = f(db.rhostore), f(db.jacobian)
        d.npml_edge, d.pml_edge_iglob = len(pm["bnd_el"]), i(pm["bnd_el"])
        d.pml_dt = float(pm["dt"])
        if at is not None and "visco" in pm and np.any(pm["visco"]):
            # attenuating layer elements: the Zener parameters of the viscoelastic CPML update
            d.pml_visco = i(pm["visco"])
            d.att_itau1, d.att_phi1 = f(at["itau1"]), f(at["phi1"])
            d.att_itau2, d.att_phi2 = f(at["itau2"]), f(at["phi2"])
            d.att_teps1, d.att_teps2 = f(at["teps1"]), f(at["teps2"])
            d.att_mu1, d.att_mu2 = f(at["mu1"]), f(at["mu2"])
    return d, keep


def time_desc(db, tile_elems: int = 32, threads_per_block: int = 256):
    """sf2d_elastic_desc with no element: the time stepping and GLL members of
    `db` only (the solid side of a fluid-only coupled run)."""
    keep = []

    def f(a):
        arr = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
        keep.append(arr)
        return arr.ctypes.data_as(_f)

    from .setup.solver_setup import ALPHA_LDDRK, BETA_LDDRK

    g = db.gll
    d = ElasticDesc()
    d.hprime, d.hprimewgll, d.wxgll, d.wzgll = f(g.hprime), f(g.hprimewgll), f(g.wxgll), f(g.wzgll)
    d.nstep = db.nstep
    d.deltat, d.deltatover2, d.deltatsquareover2 = (float(db.deltat), float(db.deltatover2),
                                                    float(db.deltatsquareover2))
    d.tile_elems, d.threads_per_block = tile_elems, threads_per_block
    d.time_scheme = int(db.time_scheme)
    d.nstage = int(db.stf.shape[2])
    d.alpha_lddrk, d.beta_lddrk = f(ALPHA_LDDRK), f(BETA_LDDRK)
    d.seismotype = 1
    return d, keep


class ElasticSolver:
    """Device-resident elastic solver (Newmark or LDDRK) for one Database."""

    def __init__(self, db, tile_elems: int = 32, seismotype: int = 1, threads_per_block: int = 256,
                 pml_tile_elems: int = 0, pml_threads_per_block: int = 0):
        lib = load_library()
        d, keep = build_desc(db, tile_elems, seismotype, threads_per_block, pml_tile_elems, pml_threads_per_block)
        h = ctypes.c_void_p()
        _check(lib.sf2d_elastic_create(ctypes.byref(d), ctypes.byref(h)))
        self._h = h
        self._lib = lib
        self.nglob = db.nglob
        self.nrec = d.nrec
        self.nstep_total = db.nstep
        del keep

    def close(self):
        if getattr(self, "_h", None):
            self._lib.sf2d_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_fields(self, displ=None, veloc=None, accel=None):
        arrs = [None if x is None else np.ascontiguousarray(x, dtype=np.float32) for x in (displ, veloc, accel)]
        ptrs = [None if x is None else x.ctypes.data_as(_f) for x in arrs]
        _check(self._lib.sf2d_set_fields(self._h, *ptrs))

    def get_fields(self, out=None):
        """displ, veloc, accel (nglob, 2); `out`: three preallocated C-contiguous float32
        arrays to fill (pinned host memory copies fastest)."""
        if out is None:
            out = [np.empty((self.nglob, 2), dtype=np.float32) for _ in range(3)]
        for a in out:
            if a.shape != (self.nglob, 2) or a.dtype != np.float32 or not a.flags.c_contiguous:
                raise ValueError(f"need C-contiguous float32 arrays of shape {(self.nglob, 2)}")
        _check(self._lib.sf2d_get_fields(self._h, *[x.ctypes.data_as(_f) for x in out]))
        return out

    def run(self, nstep: int, seismograms: bool = True, out=None):
        """Advance nstep steps; returns seismograms (nrec, nstep, 2) float64 (in `out` when
        given: a C-contiguous float64 array of that shape) or None."""
        seis = _seis_buffer(self.nrec, nstep, out) if seismograms else None
        _check(self._lib.sf2d_run(self._h, nstep, None if seis is None else seis.ctypes.data_as(_d)))
        return seis

    def enqueue(self, nstep: int):
        _check(self._lib.sf2d_enqueue(self._h, nstep))

    def prepare(self):
        """Build the step-chunk graph ahead of the first enqueue (runs nothing)."""
        _check(self._lib.sf2d_prepare(self._h))

    def synchronize(self, timeout_s: float = 0.0):
        _check(self._lib.sf2d_synchronize(self._h, float(timeout_s)))

    def set_members(self, elem_member):
        """Name the member (independent sub-mesh) of every element of a packed
        batch: a member whose field blows up is then masked and the others run on."""
        m = np.ascontiguousarray(np.asarray(elem_member, dtype=np.int32))
        self.nmembers = int(m.max()) + 1
        _check(self._lib.sf2d_set_members(self._h, m.ctypes.data_as(_i), self.nmembers))

    def member_status(self) -> np.ndarray:
        """Per member: 0 running, 1 masked (its field blew up)."""
        st = np.zeros(self.nmembers, dtype=np.int32)
        _check(self._lib.sf2d_member_status(self._h, st.ctypes.data_as(_i)))
        return st

    def copy_seismograms(self, it0: int, nstep: int, out=None):
        if out is None:
            out = np.zeros((self.nrec, nstep, 2), dtype=np.float64)
        _check(self._lib.sf2d_copy_seismograms(self._h, it0, nstep, out.ctypes.data_as(_d)))
        return out

    def max_norm(self) -> float:
        v = ctypes.c_float()
        _check(self._lib.sf2d_get_norm(self._h, ctypes.byref(v)))
        return float(v.value)

    def step_index(self) -> int:
        v = ctypes.c_int()
        _check(self._lib.sf2d_step_index(self._h, ctypes.byref(v)))
        return int(v.value)

    def stream_handle(self) -> int:
        v = ctypes.c_void_p()
        _check(self._lib.sf2d_get_stream(self._h, ctypes.byref(v)))
        return int(v.value or 0)

    def time_kernels(self, nstep: int):
        ms = (ctypes.c_float * 3)()
        _check(self._lib.sf2d_time_kernels(self._h, nstep, ms))
        return [float(x) for x in ms]

    def layout_info(self):
        v = (ctypes.c_longlong * 8)()
        _check(self._lib.sf2d_layout_info(self._h, v))
        keys = ["ntiles", "nshared", "max_local", "max_elems", "device_bytes", "smem_bytes",
                "threads_per_block", "n_slots"]
        return dict(zip(keys, [int(x) for x in v]))

    def launch_count(self, nstep: int) -> int:
        """Kernel launches that enqueue(nstep) issues."""
        n = ctypes.c_longlong()
        _check(self._lib.sf2d_launch_count(self._h, nstep, ctypes.byref(n)))
        return int(n.value)
