"""Batches of shots and of independent models advanced in one launch per step.

A batch is packed into one disconnected mesh: member m's elements, global
points, absorbing points, sources and receivers are appended with offsets
(its element ids shifted by the elements before it, its global ids by the
points before it), and its coordinates are shifted far apart along x so the
Morton-ordered tiles of the tiler never mix members.  The tile-staged kernels
need no change: every tile belongs to one member, shared points stay inside a
member, and the per-step launch count is that of a single run.  This is the
GPU counterpart of the reference's NUMBER_OF_SIMULTANEOUS_RUNS
(src/shared/parallel.F90:40-50, 1714), which runs independent simulations as
separate MPI groups.

Members must share the time step and the number of steps.  Seismograms come
back per member; kernels of a gradient batch are returned per member (or
summed over the shots of one model).
"""
from __future__ import annotations

import copy
import dataclasses

import numpy as np

from .setup.solver_setup import Database

SHIFT = 1.0e8  # metres between consecutive members along x


@dataclasses.dataclass
class BatchIndex:
    elem_off: np.ndarray   # (M+1,) element offsets
    glob_off: np.ndarray   # (M+1,) global point offsets
    rec_off: np.ndarray    # (M+1,) receiver offsets


def pack(members) -> tuple[Database, BatchIndex]:
    """Concatenate Databases (same dt, nstep, time scheme) into one."""
    if not members:
        raise ValueError("empty batch")
    d0 = members[0]
    for d in members[1:]:
        if float(d.dt) != float(d0.dt) or d.nstep != d0.nstep or d.time_scheme != d0.time_scheme:
            raise ValueError("batch members must share dt, nstep and the time scheme")
        if (d.atten is None) != (d0.atten is None) or (d.aniso is None) != (d0.aniso is None):
            raise ValueError("batch members must share the physics (attenuation, anisotropy)")
    for d in members:
        # the packed mesh concatenates the solid arrays only
        if getattr(d, "acoustic", None) is not None or getattr(d, "pml", None) is not None:
            raise ValueError("batch members with fluid elements or CPML layers cannot be packed")
    eo = np.cumsum([0] + [d.nspec for d in members])
    go = np.cumsum([0] + [d.nglob for d in members])
    ro = np.cumsum([0] + [len(d.rec_ispec) for d in members])

    def cat(name, shift=None):
        parts = []
        for m, d in enumerate(members):
            a = getattr(d, name)
            if shift == "glob":
                a = a + go[m]
            elif shift == "elem":
                a = a + eo[m]
            parts.append(a)
        return np.concatenate(parts, axis=0)

    coord = np.concatenate([d.coord + np.array([m * SHIFT, 0.0]) for m, d in enumerate(members)], axis=0)
    nstage = d0.stf.shape[2]
    out = copy.copy(d0)
    out.nspec = int(eo[-1])
    out.nglob = int(go[-1])
    out.ibool = cat("ibool", "glob").astype(np.int32)
    for name in ("xix", "xiz", "gammax", "gammaz", "jacobian", "rhostore", "kappastore", "mustore",
                 "rho_vpstore", "rho_vsstore", "rmass_inverse_elastic", "stacey_nx", "stacey_nz",
                 "stacey_weight", "stacey_rho_vp", "stacey_rho_vs", "sourcearrays", "hxir", "hgammar",
                 "rec_xi", "rec_gamma", "rec_x", "rec_z"):
        setattr(out, name, cat(name))
    out.coord = coord
    out.stacey_iglob = cat("stacey_iglob", "glob").astype(np.int32)
    out.source_ispec = cat("source_ispec", "elem").astype(np.int32)
    out.rec_ispec = cat("rec_ispec", "elem").astype(np.int32)
    out.stf = np.concatenate([d.stf.reshape(-1, d.nstep, nstage) for d in members], axis=0)
    if d0.atten is not None:
        out.atten = {k: np.concatenate([d.atten[k] for d in members], axis=0) for k in d0.atten}
    if d0.aniso is not None:
        out.aniso = {k: np.concatenate([d.aniso[k] for d in members], axis=0) for k in d0.aniso}
    out.mesh = None
    return out, BatchIndex(eo, go, ro)


def split_seismograms(seis, index: BatchIndex):
    """Per-member views of batched receiver traces (nrec_total, nstep, 2)."""
    return [seis[index.rec_off[m]:index.rec_off[m + 1]] for m in range(len(index.rec_off) - 1)]


def element_members(index: BatchIndex) -> np.ndarray:
    """Member id of every element of a packed Database (for ElasticSolver.set_members)."""
    off = np.asarray(index.elem_off)
    return np.repeat(np.arange(len(off) - 1, dtype=np.int32), np.diff(off))


def split_elements(arr, index: BatchIndex):
    """Per-member views of a per-element array (nspec_total, ...)."""
    return [arr[index.elem_off[m]:index.elem_off[m + 1]] for m in range(len(index.elem_off) - 1)]


def shots_on_model(db, positions, angle_deg: float = 0.0):
    """Copies of `db` that differ only in the position of its force source.

    The source arrays are recomputed at each (x, z) with the setup's point
    location (locate_source.F90) and the force angle `angle_deg`
    (setup_sources_receivers.F90:993-1010); the time function is kept.
    """
    import math

    from .setup.gll import NGLL, lagrange_any
    from .setup.solver_setup import _locate, _PointLocator

    if db.mesh is None:
        raise ValueError("needs the mesh the database was built from")
    locator = _PointLocator(db.ibool, db.coord)
    ang = angle_deg * math.pi / 180.0
    out = []
    for (xs, zs) in positions:
        e, xi, gamma, _, _ = _locate(db.mesh, db.ibool, db.coord, db.gll, xs, zs, iterate=True, locator=locator)
        hx, _ = lagrange_any(xi, db.gll.xigll)
        hg, _ = lagrange_any(gamma, db.gll.zigll)
        arr = np.zeros((NGLL, NGLL, 2), dtype=np.float32)
        for j in range(NGLL):
            for i in range(NGLL):
                h = hx[i] * hg[j]
                arr[j, i, 0] = np.float32(math.sin(ang) * h)
                arr[j, i, 1] = np.float32(-math.cos(ang) * h)
        d = copy.copy(db)
        d.source_ispec = np.array([e], dtype=np.int32)
        d.sourcearrays = arr.reshape(1, NGLL, NGLL, 2)
        d.stf = db.stf[:1].copy()
        d.src_xi = np.array([xi])
        d.src_gamma = np.array([gamma])
        out.append(d)
    return out


class NativeBatch:
    """A batch packed by the library itself (sf2d_batch_*, include/sf2d_b200.h):
    the models' descriptions and, optionally, shots on them (each a Database
    of one of the models that differs only in its sources, as shots_on_model
    makes them).  checkpoint_every > 0 makes a gradient batch whose kernels
    come back per model, summed over its shots."""

    def __init__(self, models, shots=None, shot_models=None, checkpoint_every: int = 0, tile_elems: int = 32,
                 threads_per_block: int = 256):
        import ctypes

        from .runtime import ElasticDesc, _check, build_desc, load_library

        lib = load_library()
        vp, ip = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)
        fp = ctypes.POINTER(ctypes.c_float)

        class Shot(ctypes.Structure):
            _fields_ = [("model", ctypes.c_int), ("nsrc", ctypes.c_int), ("src_ispec", ip),
                        ("sourcearrays", fp), ("stf", fp)]

        lib.sf2d_batch_create.argtypes = [ctypes.POINTER(ElasticDesc), ctypes.c_int, ctypes.POINTER(Shot),
                                          ctypes.c_int, ctypes.POINTER(fp), ctypes.POINTER(fp), ctypes.c_int,
                                          ctypes.POINTER(vp)]
        for name, args in (("sf2d_batch_info", [vp, ctypes.POINTER(ctypes.c_longlong)]),
                           ("sf2d_batch_run_forward", [vp, ctypes.POINTER(ctypes.c_double)]),
                           ("sf2d_batch_run_adjoint", [vp, fp, fp, fp, fp]),
                           ("sf2d_batch_member_status", [vp, ip]), ("sf2d_batch_destroy", [vp])):
            getattr(lib, name).argtypes = args
        self._lib, self._keep = lib, []
        descs = (ElasticDesc * len(models))()
        for k, db in enumerate(models):
            d, keep = build_desc(db, tile_elems, 1, threads_per_block)
            descs[k] = d
            self._keep.append(keep)
        shots = list(shots or [])
        shot_arr = (Shot * max(len(shots), 1))()
        for s, db in enumerate(shots):
            ispec = np.ascontiguousarray(db.source_ispec, dtype=np.int32)
            arr = np.ascontiguousarray(db.sourcearrays, dtype=np.float32)
            stf = np.ascontiguousarray(db.stf, dtype=np.float32)
            self._keep.append((ispec, arr, stf))
            shot_arr[s] = Shot(int(shot_models[s]) if shot_models is not None else 0, len(ispec),
                               ispec.ctypes.data_as(ip), arr.ctypes.data_as(fp), stf.ctypes.data_as(fp))
        rho = (fp * len(models))()
        kap = (fp * len(models))()
        if checkpoint_every:
            for k, db in enumerate(models):
                r = np.ascontiguousarray(db.rhostore, dtype=np.float32)
                q = np.ascontiguousarray(db.kappastore, dtype=np.float32)
                self._keep.append((r, q))
                rho[k], kap[k] = r.ctypes.data_as(fp), q.ctypes.data_as(fp)
        h = vp()
        _check(lib.sf2d_batch_create(descs, len(models), shot_arr, len(shots), rho, kap, int(checkpoint_every),
                                     ctypes.byref(h)))
        self._h = h
        info = (ctypes.c_longlong * 4)()
        _check(lib.sf2d_batch_info(h, info))
        self.nmembers, self.nspec, self.nglob, self.nrec = (int(x) for x in info)
        self.nstep = int(models[0].nstep)
        self.model_nspec = [int(db.nspec) for db in models]

    def forward(self) -> np.ndarray:
        """Seismograms of all members (nrec_total, nstep, 2), members in order."""
        from .runtime import _check, _d

        seis = np.zeros((self.nrec, self.nstep, 2), dtype=np.float64)
        _check(self._lib.sf2d_batch_run_forward(self._h, seis.ctypes.data_as(_d)))
        return seis

    def adjoint(self, adj_src):
        """Kernels (rho, kappa, mu) of each model, (nspec, 5, 5) each, summed over its shots."""
        from .runtime import _check, _f

        adj = np.ascontiguousarray(np.asarray(adj_src, dtype=np.float32).reshape(self.nrec, self.nstep, 2))
        n = sum(self.model_nspec)
        out = [np.zeros((n, 5, 5), dtype=np.float32) for _ in range(3)]
        _check(self._lib.sf2d_batch_run_adjoint(self._h, adj.ctypes.data_as(_f),
                                                *[o.ctypes.data_as(_f) for o in out]))
        off = np.cumsum([0] + self.model_nspec)
        return [tuple(o[off[k]:off[k + 1]] for o in out) for k in range(len(self.model_nspec))]

    def member_status(self) -> np.ndarray:
        import ctypes

        from .runtime import _check

        st = np.zeros(self.nmembers, dtype=np.int32)
        _check(self._lib.sf2d_batch_member_status(self._h, st.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))
        return st

    def close(self):
        if getattr(self, "_h", None):
            self._lib.sf2d_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
