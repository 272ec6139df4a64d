"""Coupled fluid-solid runs on the GPU.

A Database with acoustic elements is split into a solid sub-mesh (handed to
the elastic tile solver unchanged) and a fluid sub-mesh (the acoustic tile
solver), each with its own compact numbering of the points it touches.  The
fluid-solid interface points exist in both numberings; the coupling lists
name them in both.  ``CoupledSolver`` wraps sf2d_coupled_* of the C ABI
(include/sf2d_coupled.h) and gives fields and seismograms back in the
Database's global numbering and receiver order.
"""
from __future__ import annotations

import copy
import ctypes

import numpy as np

from .runtime import _check, _d, _f, _i, _seis_buffer, build_desc, load_library, time_desc

_vp = ctypes.c_void_p


class AcousticDesc(ctypes.Structure):
    _fields_ = [
        ("nspec", ctypes.c_int), ("nglob", ctypes.c_int),
        ("ibool", _i),
        ("xix", _f), ("xiz", _f), ("gammax", _f), ("gammaz", _f),
        ("jacobian", _f), ("rhostore", _f), ("kappastore", _f),
        ("rmass_inverse", _f),
        ("centroid_xz", _d),
        ("nfree", ctypes.c_int), ("free_iglob", _i),
        ("nstacey", ctypes.c_int), ("st_iglob", _i), ("st_w", _f), ("st_rho_vp", _f),
        ("nsrc", ctypes.c_int), ("src_ispec", _i), ("sourcearrays", _f), ("stf", _f),
        ("nrec", ctypes.c_int), ("rec_ispec", _i), ("hxir", _d), ("hgammar", _d), ("rec_global", _i),
        ("tile_elems", ctypes.c_int),
        ("pml_region", _i),
        ("pml_K_x", _d), ("pml_K_z", _d), ("pml_d_x", _d), ("pml_d_z", _d), ("pml_alpha_x", _d), ("pml_alpha_z", _d),
        ("npml_edge", ctypes.c_int), ("pml_edge_iglob", _i),
        ("pml_dt", ctypes.c_double),
        ("threads_per_block", ctypes.c_int),
    ]


class CouplingDesc(ctypes.Structure):
    _fields_ = [
        ("nrec_total", ctypes.c_int), ("el_rec_global", _i),
        ("seismotype", ctypes.c_int), ("use_trick", ctypes.c_int),
        ("cosrot", ctypes.c_double), ("sinrot", ctypes.c_double),
        ("ncpl_ac", ctypes.c_int), ("cpl_ac_point", _i), ("cpl_ac_el_point", _i),
        ("cpl_ac_nx", _f), ("cpl_ac_nz", _f), ("cpl_ac_w", _f),
        ("ncpl_el", ctypes.c_int), ("cpl_el_point", _i), ("cpl_el_ac_point", _i),
        ("cpl_el_nx", _f), ("cpl_el_nz", _f), ("cpl_el_w", _f),
        ("cpl_ac_el_elpt", _i), ("cpl_el_ac_elpt", _i),
        ("adjoint", ctypes.c_int),
    ]


def _lib():
    from .runtime import ElasticDesc

    lib = load_library()
    if not getattr(lib, "_coupled_sigs", False):
        lib.sf2d_coupled_create.argtypes = [ctypes.POINTER(ElasticDesc), ctypes.POINTER(AcousticDesc),
                                            ctypes.POINTER(CouplingDesc), ctypes.POINTER(_vp)]
        lib.sf2d_coupled_run.argtypes = [_vp, ctypes.c_int, _d]
        lib.sf2d_coupled_get_fields.argtypes = [_vp, _f, _f, _f, _f, _f, _f]
        lib.sf2d_coupled_set_fields.argtypes = [_vp, _f, _f, _f, _f, _f, _f]
        lib.sf2d_coupled_time_kernels.argtypes = [_vp, ctypes.c_int, _f]
        lib.sf2d_coupled_layout_info.argtypes = [_vp, ctypes.POINTER(ctypes.c_longlong)]
        lib.sf2d_coupled_destroy.argtypes = [_vp]
        lib.sf2d_coupled_enqueue.argtypes = [_vp, ctypes.c_int]
        lib.sf2d_coupled_prepare.argtypes = [_vp]
        lib.sf2d_coupled_synchronize.argtypes = [_vp]
        lib.sf2d_coupled_get_stream.argtypes = [_vp, ctypes.POINTER(_vp)]
        lib.sf2d_coupled_solid_layout_info.argtypes = [_vp, ctypes.POINTER(ctypes.c_longlong)]
        lib.sf2d_coupled_launch_count.argtypes = [_vp, ctypes.c_int, ctypes.POINTER(ctypes.c_longlong)]
        lib.sf2d_coupled_set_global_numbering.argtypes = [_vp, ctypes.c_int, _i, _i]
        lib.sf2d_coupled_set_fields_global.argtypes = [_vp, _f, _f, _f, _f, _f, _f]
        lib.sf2d_coupled_get_fields_global.argtypes = [_vp, _f, _f, _f, _f, _f, _f]
        for n in ("create", "run", "get_fields", "set_fields", "time_kernels", "layout_info", "destroy",
                  "enqueue", "synchronize", "get_stream", "solid_layout_info", "launch_count", "prepare"):
            getattr(lib, "sf2d_coupled_" + n).restype = ctypes.c_int
        lib._coupled_sigs = True
    return lib


def _submesh(db, elems):
    """Sorted global ids of the points of ``elems``, global -> local map, element map."""
    pts = np.unique(db.ibool[elems])
    gmap = np.full(db.nglob, -1, dtype=np.int64)
    gmap[pts] = np.arange(len(pts))
    emap = np.full(db.nspec, -1, dtype=np.int64)
    emap[elems] = np.arange(len(elems))
    return pts, gmap, emap


def _fluid_arrays(db, ac_e, src_ac, rec_ac, pml_keys):
    """The fluid sub-mesh of the acoustic elements ac_e: its arrays (compact
    point numbering), its global points, and the point and element maps."""
    ac = db.acoustic
    pm = getattr(db, "pml", None)
    ga, amap, eamap = _submesh(db, ac_e)
    fluid = dict(
        nspec=len(ac_e), nglob=len(ga), ibool=amap[db.ibool[ac_e]].astype(np.int32),
        xix=db.xix[ac_e], xiz=db.xiz[ac_e], gammax=db.gammax[ac_e], gammaz=db.gammaz[ac_e],
        jacobian=db.jacobian[ac_e], rhostore=db.rhostore[ac_e], kappastore=db.kappastore[ac_e],
        rmass=ac["rmass"][ga], centroid=db.coord[db.ibool[ac_e][:, [0, 0, 4, 4], [0, 4, 0, 4]]].mean(axis=1),
        free=amap[ac["free_iglob"]].astype(np.int32),
        st_iglob=amap[ac["st_iglob"]].astype(np.int32), st_w=ac["st_w"], st_rvp=ac["st_rvp"],
        src_ispec=eamap[db.source_ispec[src_ac]].astype(np.int32),
        sourcearrays=db.sourcearrays[src_ac][..., 0].astype(np.float32), stf=db.stf[src_ac],
        rec_ispec=eamap[db.rec_ispec[rec_ac]].astype(np.int32), hxir=db.hxir[rec_ac], hgammar=db.hgammar[rec_ac],
        rec_global=np.flatnonzero(rec_ac).astype(np.int32), pml=None)
    if pm is not None:
        bnd_ac = amap[np.asarray(pm["bnd_ac"], dtype=np.int64)]
        fluid["pml"] = dict(region=np.asarray(pm["region"])[ac_e], bnd=bnd_ac[bnd_ac >= 0].astype(np.int32),
                            dt=pm["dt"], **{k: pm[k][ac_e] for k in pml_keys})
    return fluid, ga, amap, eamap


def split(db):
    """Return (solid Database, fluid arrays dict, coupling arrays dict, index maps)."""
    ac = db.acoustic
    if ac is None:
        raise ValueError("the Database has no acoustic element")
    pm = getattr(db, "pml", None)
    is_ac = np.asarray(ac["ispec"], dtype=bool)
    el_e, ac_e = np.flatnonzero(~is_ac), np.flatnonzero(is_ac)
    src_ac = is_ac[db.source_ispec]
    rec_ac = is_ac[db.rec_ispec]
    pml_keys = ("K_x", "K_z", "d_x", "d_z", "alpha_x", "alpha_z")
    fluid, ga, amap, eamap = _fluid_arrays(db, ac_e, src_ac, rec_ac, pml_keys)
    if len(el_e) == 0:
        # fluid-only mesh: no solid sub-mesh, no coupling
        e, ef = np.zeros(0, np.int32), np.zeros(0, np.float32)
        cpl = dict(el_rec_global=e, ac_point=e, ac_el_point=e, ac_nx=ef, ac_nz=ef, ac_w=ef, el_point=e,
                   el_ac_point=e, el_nx=ef, el_nz=ef, el_w=ef, use_trick=bool(ac.get("use_trick", False)),
                   ac_el_elpt=None, el_ac_elpt=None)
        return None, fluid, cpl, dict(solid_points=np.zeros(0, np.int64), fluid_points=ga)
    gl, gmap, emap = _submesh(db, el_e)

    sub = copy.copy(db)
    sub.nspec, sub.nglob = len(el_e), len(gl)
    sub.ibool = gmap[db.ibool[el_e]].astype(np.int32)
    for k in ("xix", "xiz", "gammax", "gammaz", "jacobian", "rhostore", "kappastore", "mustore",
              "rho_vpstore", "rho_vsstore"):
        setattr(sub, k, getattr(db, k)[el_e])
    sub.coord = db.coord[gl]
    sub.rmass_inverse_elastic = db.rmass_inverse_elastic[gl]
    sub.stacey_iglob = gmap[db.stacey_iglob].astype(np.int32)
    if (sub.stacey_iglob < 0).any():
        raise ValueError("solid absorbing point outside the solid sub-mesh")
    sm = ~src_ac
    sub.source_ispec = emap[db.source_ispec[sm]].astype(np.int32)
    sub.sourcearrays = db.sourcearrays[sm]
    sub.stf = db.stf[sm]
    rm = ~rec_ac
    sub.rec_ispec = emap[db.rec_ispec[rm]].astype(np.int32)
    sub.hxir, sub.hgammar = db.hxir[rm], db.hgammar[rm]
    if db.atten is not None:
        sub.atten = {k: v[el_e] for k, v in db.atten.items()}
    if db.aniso is not None:
        sub.aniso = {k: v[el_e] for k, v in db.aniso.items()}
    sub.acoustic = None
    sub.mesh = None
    if pm is not None:
        bnd_el = gmap[np.asarray(pm["bnd_el"], dtype=np.int64)]
        sub.pml = dict(region=np.asarray(pm["region"])[el_e], bnd_el=bnd_el[bnd_el >= 0].astype(np.int32),
                       bnd_ac=np.zeros(0, np.int32), dt=pm["dt"], **{k: pm[k][el_e] for k in pml_keys})

    cpl = dict(
        el_rec_global=np.flatnonzero(~rec_ac).astype(np.int32),
        ac_point=amap[ac["cpl_ac_iglob"]].astype(np.int32), ac_el_point=gmap[ac["cpl_ac_iglob"]].astype(np.int32),
        ac_nx=ac["cpl_ac_nx"], ac_nz=ac["cpl_ac_nz"], ac_w=ac["cpl_ac_w"],
        el_point=gmap[ac["cpl_el_iglob"]].astype(np.int32), el_ac_point=amap[ac["cpl_el_iglob"]].astype(np.int32),
        el_nx=ac["cpl_el_nx"], el_nz=ac["cpl_el_nz"], el_w=ac["cpl_el_w"],
        use_trick=bool(ac.get("use_trick", False)), ac_el_elpt=None, el_ac_elpt=None)
    if "cpl_ac_elpt" in ac:
        # element GLL points behind each entry, in the sub-mesh element numberings
        q = np.asarray(ac["cpl_ac_elpt"], dtype=np.int64)
        cpl["ac_el_elpt"] = (emap[q // 25] * 25 + q % 25).astype(np.int32)
        q = np.asarray(ac["cpl_el_acpt"], dtype=np.int64)
        cpl["el_ac_elpt"] = (eamap[q // 25] * 25 + q % 25).astype(np.int32)
        if (cpl["ac_el_elpt"] < 0).any() or (cpl["el_ac_elpt"] < 0).any():
            raise ValueError("coupling entry behind an element of the wrong domain")
    return sub, fluid, cpl, dict(solid_points=gl, fluid_points=ga)


def coupled_descs(db, tile_elems: int = 32, threads_per_block: int = 256, fluid_tile_elems: int = 0,
                  fluid_threads_per_block: int = 0, pml_tile_elems: int = 0, pml_threads_per_block: int = 0):
    """The C descriptions of a coupled Database: (solid desc, fluid desc,
    coupling desc, arrays to keep alive, solid sub-Database or None, fluid
    arrays, coupling arrays, point maps)."""
    sub, fl, cp, maps = split(db)
    seismotype = int(getattr(db, "seismotype", 1))
    if sub is not None:
        ed, keep = build_desc(sub, tile_elems, 1 if seismotype in (4, 6) else seismotype, threads_per_block,
                              pml_tile_elems, pml_threads_per_block)
    else:  # fluid-only mesh
        ed, keep = time_desc(db, tile_elems, threads_per_block)

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

    a = AcousticDesc()
    a.nspec, a.nglob = fl["nspec"], fl["nglob"]
    a.ibool = i(fl["ibool"])
    a.xix, a.xiz, a.gammax, a.gammaz = f(fl["xix"]), f(fl["xiz"]), f(fl["gammax"]), f(fl["gammaz"])
    a.jacobian, a.rhostore, a.kappastore = f(fl["jacobian"]), f(fl["rhostore"]), f(fl["kappastore"])
    a.rmass_inverse = f(fl["rmass"])
    a.centroid_xz = dd(fl["centroid"])
    a.nfree, a.free_iglob = len(fl["free"]), i(fl["free"])
    a.nstacey, a.st_iglob = len(fl["st_iglob"]), i(fl["st_iglob"])
    a.st_w, a.st_rho_vp = f(fl["st_w"]), f(fl["st_rvp"])
    a.nsrc, a.src_ispec = len(fl["src_ispec"]), i(fl["src_ispec"])
    a.sourcearrays, a.stf = f(fl["sourcearrays"]), f(fl["stf"])
    a.nrec, a.rec_ispec = len(fl["rec_ispec"]), i(fl["rec_ispec"])
    a.hxir, a.hgammar, a.rec_global = dd(fl["hxir"]), dd(fl["hgammar"]), i(fl["rec_global"])
    a.tile_elems = fluid_tile_elems or tile_elems
    a.threads_per_block = fluid_threads_per_block
    fp = fl["pml"]
    if fp is not None:
        a.pml_region = i(fp["region"])
        a.pml_K_x, a.pml_K_z = dd(fp["K_x"]), dd(fp["K_z"])
        a.pml_d_x, a.pml_d_z = dd(fp["d_x"]), dd(fp["d_z"])
        a.pml_alpha_x, a.pml_alpha_z = dd(fp["alpha_x"]), dd(fp["alpha_z"])
        a.npml_edge, a.pml_edge_iglob = len(fp["bnd"]), i(fp["bnd"])
        a.pml_dt = float(fp["dt"])
    c = CouplingDesc()
    c.nrec_total = len(db.rec_ispec)
    c.el_rec_global = i(cp["el_rec_global"])
    c.seismotype, c.use_trick = seismotype, int(cp["use_trick"])
    c.cosrot, c.sinrot = float(db.cosrot), float(db.sinrot)
    c.ncpl_ac = len(cp["ac_point"])
    c.cpl_ac_point, c.cpl_ac_el_point = i(cp["ac_point"]), i(cp["ac_el_point"])
    c.cpl_ac_nx, c.cpl_ac_nz, c.cpl_ac_w = f(cp["ac_nx"]), f(cp["ac_nz"]), f(cp["ac_w"])
    c.ncpl_el = len(cp["el_point"])
    c.cpl_el_point, c.cpl_el_ac_point = i(cp["el_point"]), i(cp["el_ac_point"])
    c.cpl_el_nx, c.cpl_el_nz, c.cpl_el_w = f(cp["el_nx"]), f(cp["el_nz"]), f(cp["el_w"])
    if cp["ac_el_elpt"] is not None:
        c.cpl_ac_el_elpt, c.cpl_el_ac_elpt = i(cp["ac_el_elpt"]), i(cp["el_ac_elpt"])
    return ed, a, c, keep, sub, fl, cp, maps


class CoupledSolver:
    """Device-resident coupled fluid-solid solver for one Database."""

    def __init__(self, db, tile_elems: int = 32, threads_per_block: int = 256, fluid_tile_elems: int = 0,
                 fluid_threads_per_block: int = 0, pml_tile_elems: int = 0, pml_threads_per_block: int = 0):
        """Tile sizes and threads per CTA of the solid; the fluid's default to the same."""
        lib = _lib()
        ed, a, c, keep, sub, fl, cp, maps = coupled_descs(db, tile_elems, threads_per_block, fluid_tile_elems,
                                                          fluid_threads_per_block, pml_tile_elems,
                                                          pml_threads_per_block)
        h = _vp()
        _check(lib.sf2d_coupled_create(ctypes.byref(ed), ctypes.byref(a), ctypes.byref(c), ctypes.byref(h)))
        self._h, self._lib = h, lib
        self.nglob, self.nrec, self.nstep_total = db.nglob, len(db.rec_ispec), db.nstep
        self.solid_points, self.fluid_points = maps["solid_points"], maps["fluid_points"]
        # whole-mesh numbering on the device: field transfers permute there
        sp = None if sub is None else np.ascontiguousarray(self.solid_points, dtype=np.int32)
        fp = np.ascontiguousarray(self.fluid_points, dtype=np.int32)
        _check(lib.sf2d_coupled_set_global_numbering(h, int(db.nglob), None if sp is None else sp.ctypes.data_as(_i),
                                                     fp.ctypes.data_as(_i)))
        self.sub_db = sub
        self.nspec_fluid, self.nglob_fluid = fl["nspec"], fl["nglob"]
        del keep

    def close(self):
        if getattr(self, "_h", None):
            self._lib.sf2d_coupled_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, nstep: int, seismograms: bool = True, out=None):
        """Advance nstep steps; returns seismograms (nrec, nstep, 2) float64 (in `out` when
        given: a C-contiguous float64 array of that shape) or None."""
        seis = _seis_buffer(self.nrec, nstep, out) if seismograms else None
        _check(self._lib.sf2d_coupled_run(self._h, nstep, None if seis is None else seis.ctypes.data_as(_d)))
        return seis

    def enqueue(self, nstep: int):
        _check(self._lib.sf2d_coupled_enqueue(self._h, nstep))

    def prepare(self):
        """Build the step-chunk graph ahead of the first enqueue (runs nothing)."""
        _check(self._lib.sf2d_coupled_prepare(self._h))

    def synchronize(self, timeout_s: float = 0.0):
        _check(self._lib.sf2d_coupled_synchronize(self._h))

    def stream_handle(self) -> int:
        v = _vp()
        _check(self._lib.sf2d_coupled_get_stream(self._h, ctypes.byref(v)))
        return int(v.value or 0)

    def get_fields(self, out=None):
        """displ, veloc, accel (nglob, 2) and pot, pot_dot, pot_dot_dot (nglob,) in global numbering
        (points outside a field's domain read zero).  `out`: a dict of preallocated float32
        C-contiguous arrays to fill (pinned host memory copies fastest)."""
        shapes = {"displ": (self.nglob, 2), "veloc": (self.nglob, 2), "accel": (self.nglob, 2),
                  "pot": (self.nglob,), "pot_dot": (self.nglob,), "pot_dot_dot": (self.nglob,)}
        res = {}
        for k, shp in shapes.items():
            a = None if out is None else out.get(k)
            if a is None:
                a = np.empty(shp, dtype=np.float32)
            elif a.shape != shp or a.dtype != np.float32 or not a.flags.c_contiguous:
                raise ValueError(f"{k}: need a C-contiguous float32 array of shape {shp}")
            res[k] = a
        _check(self._lib.sf2d_coupled_get_fields_global(
            self._h, *[res[k].ctypes.data_as(_f) for k in shapes]))
        return res

    def set_fields(self, **fields):
        """Set displ/veloc/accel (nglob, 2) and pot/pot_dot/pot_dot_dot (nglob,) (global numbering);
        missing fields are zeroed.  Arrays are used in place when they are C-contiguous float32."""
        ptrs, keep = [], []
        for k, shp in (("displ", (self.nglob, 2)), ("veloc", (self.nglob, 2)), ("accel", (self.nglob, 2)),
                       ("pot", (self.nglob,)), ("pot_dot", (self.nglob,)), ("pot_dot_dot", (self.nglob,))):
            v = fields.get(k)
            if v is None:
                ptrs.append(None)
                continue
            a = np.ascontiguousarray(v, dtype=np.float32)
            if a.shape != shp:
                raise ValueError(f"{k}: expected shape {shp}, got {a.shape}")
            keep.append(a)
            ptrs.append(a.ctypes.data_as(_f))
        _check(self._lib.sf2d_coupled_set_fields_global(self._h, *ptrs))

    def time_kernels(self, nstep: int):
        """Average ms per launch: fluid tile, fluid shared, solid tile, solid shared; and per step."""
        ms = (ctypes.c_float * 5)()
        _check(self._lib.sf2d_coupled_time_kernels(self._h, nstep, ms))
        return [float(x) for x in ms]

    def layout_info(self):
        """Layout of the fluid tiling."""
        info = (ctypes.c_longlong * 6)()
        _check(self._lib.sf2d_coupled_layout_info(self._h, info))
        keys = ["ntiles", "nshared", "max_local", "smem", "n_interior", "n_slots"]
        return dict(zip(keys, [int(x) for x in info]))

    def solid_layout_info(self):
        """Layout of the solid tiling (keys of ElasticSolver.layout_info)."""
        v = (ctypes.c_longlong * 8)()
        _check(self._lib.sf2d_coupled_solid_layout_info(self._h, v))
        keys = ["ntiles", "nshared", "max_local", "max_elems", "device_bytes", "smem_bytes",
                "threads_per_block", "n_slots"]
        return dict(zip(keys, [int(x) for x in v]))

    def launch_count(self, nstep: int) -> int:
        """Kernel launches that enqueue(nstep) issues."""
        n = ctypes.c_longlong()
        _check(self._lib.sf2d_coupled_launch_count(self._h, nstep, ctypes.byref(n)))
        return int(n.value)


def _fwi_lib():
    from .runtime import ElasticDesc

    lib = _lib()
    if not getattr(lib, "_coupled_fwi_sigs", False):
        lib.sf2d_coupled_fwi_create.argtypes = [ctypes.POINTER(ElasticDesc), ctypes.POINTER(AcousticDesc),
                                                ctypes.POINTER(CouplingDesc), _f, _f, ctypes.c_int,
                                                ctypes.POINTER(_vp)]
        lib.sf2d_coupled_fwi_forward.argtypes = [_vp, _d]
        lib.sf2d_coupled_fwi_backward.argtypes = [_vp, _f, _f, _f, _f, _f, _f]
        lib.sf2d_coupled_fwi_adjoint_seismograms.argtypes = [_vp, _d]
        lib.sf2d_coupled_fwi_destroy.argtypes = [_vp]
        for n in ("create", "forward", "backward", "adjoint_seismograms", "destroy"):
            getattr(lib, "sf2d_coupled_fwi_" + n).restype = ctypes.c_int
        lib._coupled_fwi_sigs = True
    return lib


class CoupledKernels:
    """Kernel run (SIMULATION_TYPE = 3) of a Database with fluid elements on the
    GPU (sf2d_coupled_fwi_* of the C ABI): `forward()` runs from rest with a
    state checkpoint every `checkpoint_every` steps and returns the receiver
    traces; `backward(adj_src)` runs the adjoint sweep driven by the adjoint
    sources (nrec, nstep, 2) in time order (a fluid receiver uses component 0)
    and returns the kernels in the Database's element layout:

    * ``rho``, ``kappa``, ``mu``: solid kernels scaled as save_adjoint_kernels.f90:134-141
      (zero in fluid elements);
    * ``rho_ac``, ``kappa_ac``: fluid kernels of compute_kernels.f90:420-436, deltat
      included (zero in solid elements).

    Newmark, Stacey or free edges (no CPML)."""

    def __init__(self, db, checkpoint_every: int = 200, tile_elems: int = 32, threads_per_block: int = 256):
        if int(db.time_scheme) != 1:
            raise ValueError("the kernel run is implemented for the Newmark scheme")
        if getattr(db, "pml", None) is not None:
            raise ValueError("the kernel run is implemented without CPML layers")
        lib = _fwi_lib()
        ed, a, c, keep, sub, fl, cp, maps = coupled_descs(db, tile_elems, threads_per_block)
        is_ac = np.asarray(db.acoustic["ispec"], dtype=bool)
        self.el_e, self.ac_e = np.flatnonzero(~is_ac), np.flatnonzero(is_ac)
        rho = kap = None
        if sub is not None:
            rho = np.ascontiguousarray(sub.rhostore, dtype=np.float32)
            kap = np.ascontiguousarray(sub.kappastore, dtype=np.float32)
            keep += [rho, kap]
        h = _vp()
        _check(lib.sf2d_coupled_fwi_create(ctypes.byref(ed), ctypes.byref(a), ctypes.byref(c),
                                           None if rho is None else rho.ctypes.data_as(_f),
                                           None if kap is None else kap.ctypes.data_as(_f),
                                           int(checkpoint_every), ctypes.byref(h)))
        self._h, self._lib = h, lib
        self.nrec, self.nstep, self.nspec = len(db.rec_ispec), db.nstep, db.nspec
        del keep

    def close(self):
        if getattr(self, "_h", None):
            self._lib.sf2d_coupled_fwi_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def forward(self) -> np.ndarray:
        seis = np.zeros((self.nrec, self.nstep, 2), dtype=np.float64)
        _check(self._lib.sf2d_coupled_fwi_forward(self._h, seis.ctypes.data_as(_d)))
        return seis

    def backward(self, adj_src) -> dict:
        adj = np.ascontiguousarray(np.asarray(adj_src, dtype=np.float32).reshape(self.nrec, self.nstep, 2))
        ns, nf = len(self.el_e), len(self.ac_e)
        sol = [np.zeros((ns, 5, 5), dtype=np.float32) for _ in range(3)]
        flu = [np.zeros((nf, 5, 5), dtype=np.float32) for _ in range(2)]
        ptr = [None if ns == 0 else x.ctypes.data_as(_f) for x in sol] + [x.ctypes.data_as(_f) for x in flu]
        _check(self._lib.sf2d_coupled_fwi_backward(self._h, adj.ctypes.data_as(_f), *ptr))
        out = {}
        for k, v in zip(("rho", "kappa", "mu"), sol):
            full = np.zeros((self.nspec, 5, 5), dtype=np.float32)
            full[self.el_e] = v
            out[k] = full
        for k, v in zip(("rho_ac", "kappa_ac"), flu):
            full = np.zeros((self.nspec, 5, 5), dtype=np.float32)
            full[self.ac_e] = v
            out[k] = full
        return out

    def adjoint_seismograms(self) -> np.ndarray:
        """Receiver traces (nrec, nstep, 2) of the adjoint field of the last backward()."""
        seis = np.zeros((self.nrec, self.nstep, 2), dtype=np.float64)
        _check(self._lib.sf2d_coupled_fwi_adjoint_seismograms(self._h, seis.ctypes.data_as(_d)))
        return seis


def coupled_kernels(db, adj_src, checkpoint_every: int = 200, **kw) -> dict:
    """Forward traces, adjoint traces and kernels of one kernel run: a dict with
    ``seis``, ``adj_seis`` and the kernels of CoupledKernels.backward.  `adj_src`
    is an array (nrec, nstep, 2) or a function of the forward traces."""
    k = CoupledKernels(db, checkpoint_every, **kw)
    try:
        seis = k.forward()
        src = adj_src(seis) if callable(adj_src) else adj_src
        out = k.backward(src)
        out["seis"], out["adj_seis"] = seis, k.adjoint_seismograms()
    finally:
        k.close()
    return out
