"""ctypes binding of the CPU oracle -- TEST INFRASTRUCTURE.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.  It wraps oracle/_build/libsf2d_oracle.so (built by
oracle/Makefile) and feeds it a setup Database.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libsf2d_oracle.so")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


class OracleDb(ctypes.Structure):
    _fields_ = [
        ("nspec", ctypes.c_int), ("nglob", ctypes.c_int),
        ("ibool", _ip),
        ("xix", _dp), ("xiz", _dp), ("gammax", _dp), ("gammaz", _dp), ("jacobian", _dp),
        ("rhostore", _dp), ("kappastore", _dp), ("mustore", _dp), ("rho_vpstore", _dp), ("rho_vsstore", _dp),
        ("rmass_inverse", _dp),
        ("hprime", _dp), ("hprimewgll", _dp), ("wxgll", _dp), ("wzgll", _dp),
        ("nstacey", ctypes.c_int), ("st_iglob", _ip),
        ("st_nx", _dp), ("st_nz", _dp), ("st_w", _dp), ("st_rvp", _dp), ("st_rvs", _dp),
        ("nsrc", ctypes.c_int), ("src_ispec", _ip), ("sourcearrays", _dp), ("stf", _dp),
        ("nstep_total", ctypes.c_int), ("nstage", ctypes.c_int),
        ("nrec", ctypes.c_int), ("rec_ispec", _ip), ("hxir", _dp), ("hgammar", _dp),
        ("cosrot", ctypes.c_double), ("sinrot", ctypes.c_double),
        ("seismotype", ctypes.c_int),
        ("deltat", ctypes.c_double), ("deltatover2", ctypes.c_double), ("deltatsquareover2", ctypes.c_double),
        ("ispec_is_anisotropic", _ip),
        ("c11", _dp), ("c13", _dp), ("c15", _dp), ("c33", _dp), ("c35", _dp), ("c55", _dp),
        ("time_scheme", ctypes.c_int), ("alpha_lddrk", _dp), ("beta_lddrk", _dp),
        ("att_a1", _dp), ("att_b1", _dp), ("att_a2", _dp), ("att_b2", _dp),
        ("att_itau1", _dp), ("att_phi1", _dp), ("att_itau2", _dp), ("att_phi2", _dp),
        ("adj_src", _dp),
        ("ispec_is_acoustic", _ip), ("rmass_inverse_acoustic", _dp),
        ("nstacey_ac", ctypes.c_int), ("st_ac_iglob", _ip), ("st_ac_w", _dp), ("st_ac_rvp", _dp),
        ("nfree_ac", ctypes.c_int), ("free_ac_iglob", _ip),
        ("ncpl_ac", ctypes.c_int), ("cpl_ac_iglob", _ip), ("cpl_ac_nx", _dp), ("cpl_ac_nz", _dp), ("cpl_ac_w", _dp),
        ("ncpl_el", ctypes.c_int), ("cpl_el_iglob", _ip), ("cpl_el_nx", _dp), ("cpl_el_nz", _dp), ("cpl_el_w", _dp),
        ("use_trick", ctypes.c_int),
        ("pml_region", _ip),
        ("pml_K_x", _dp), ("pml_K_z", _dp), ("pml_d_x", _dp), ("pml_d_z", _dp), ("pml_alpha_x", _dp),
        ("pml_alpha_z", _dp),
        ("npml_bnd_el", ctypes.c_int), ("npml_bnd_ac", ctypes.c_int), ("pml_bnd_el", _ip), ("pml_bnd_ac", _ip),
        ("cpl_ac_elpt", _ip), ("cpl_el_acpt", _ip),
        ("DT", ctypes.c_double),
        ("pml_visco", _ip), ("att_teps1", _dp), ("att_teps2", _dp), ("att_mu1", _dp), ("att_mu2", _dp),
    ]


DISPL, VELOC, ACCEL, DISPL_LDDRK, VELOC_LDDRK, E1, E11, E13, ATT_OLD, RHO_KL, KAPPA_KL, MU_KL = range(12)
POT, POT_DOT, POT_DOT_DOT, POT_LDDRK, POT_DOT_LDDRK = range(12, 17)
HESS1, HESS2 = 17, 18
RHO_AC_KL, KAPPA_AC_KL = 19, 20


def build() -> str:
    """Compile the oracle library if it is missing or older than its source."""
    src = os.path.join(HERE, "sf2d_oracle.cpp")
    hdr = os.path.join(HERE, "sf2d_oracle.h")
    if (not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src)
            or os.path.getmtime(LIB_PATH) < os.path.getmtime(hdr)):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(build())
        _lib.sf2d_oracle_create.restype = ctypes.c_void_p
        _lib.sf2d_oracle_create.argtypes = [ctypes.POINTER(OracleDb), ctypes.c_int]
        _lib.sf2d_oracle_run.restype = ctypes.c_int
        _lib.sf2d_oracle_run.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, ctypes.c_int]
        for fn in (_lib.sf2d_oracle_get, _lib.sf2d_oracle_set):
            fn.restype = ctypes.c_int
            fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        _lib.sf2d_oracle_accumulate_kernels.restype = ctypes.c_int
        _lib.sf2d_oracle_accumulate_kernels.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        _lib.sf2d_oracle_accumulate_kernels_acoustic.restype = ctypes.c_int
        _lib.sf2d_oracle_accumulate_kernels_acoustic.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        _lib.sf2d_oracle_accumulate_hessian.restype = ctypes.c_int
        _lib.sf2d_oracle_accumulate_hessian.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        _lib.sf2d_oracle_set_step.restype = ctypes.c_int
        _lib.sf2d_oracle_set_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
        _lib.sf2d_oracle_destroy.restype = None
        _lib.sf2d_oracle_destroy.argtypes = [ctypes.c_void_p]
        _lib.sf2d_oracle_max_threads.restype = ctypes.c_int
    return _lib


class Oracle:
    """Holds converted arrays (kept alive) and an oracle state; runs the CPU time loop."""

    def __init__(self, db, precision: int = 4, seismotype: int | None = None, db64=None, adj_src=None):
        """``db`` supplies the FP32 setup; ``db64`` (optional) the FP64 one for precision 8.
        ``seismotype`` defaults to the database's."""
        from specfem2d_b200.setup.solver_setup import ALPHA_LDDRK, BETA_LDDRK

        self.precision = precision
        src = db64 if (precision == 8 and db64 is not None) else db
        self.db = src
        keep = []

        def d(a):
            if a is None:
                return None
            arr = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
            keep.append(arr)
            return arr.ctypes.data_as(_dp)

        def i(a):
            if a is None:
                return None
            arr = np.ascontiguousarray(np.asarray(a, dtype=np.int32))
            keep.append(arr)
            return arr.ctypes.data_as(_ip)

        g = src.gll
        if precision == 8:
            hprime = g.hprime_dble
            hprimewgll = g.wgll_dble[:, None] * g.hprime_dble
            wx = g.wgll_dble
            dt = float(src.dt)
            dto2 = 0.5 * dt
            dt2o2 = 0.5 * dt * dt
        else:
            hprime = g.hprime
            hprimewgll = g.hprimewgll
            wx = g.wxgll
            dt = float(src.deltat)
            dto2 = float(src.deltatover2)
            dt2o2 = float(src.deltatsquareover2)
        nstage = src.stf.shape[2] if src.stf.ndim == 3 else 1
        s = OracleDb()
        s.nspec, s.nglob = src.nspec, src.nglob
        s.ibool = i(src.ibool)
        s.xix, s.xiz, s.gammax, s.gammaz, s.jacobian = (d(src.xix), d(src.xiz), d(src.gammax),
                                                        d(src.gammaz), d(src.jacobian))
        s.rhostore, s.kappastore, s.mustore = d(src.rhostore), d(src.kappastore), d(src.mustore)
        s.rho_vpstore, s.rho_vsstore = d(src.rho_vpstore), d(src.rho_vsstore)
        s.rmass_inverse = d(src.rmass_inverse_elastic)
        s.hprime, s.hprimewgll, s.wxgll, s.wzgll = d(hprime), d(hprimewgll), d(wx), d(wx)
        s.nstacey = len(src.stacey_iglob)
        s.st_iglob = i(src.stacey_iglob)
        s.st_nx, s.st_nz, s.st_w = d(src.stacey_nx), d(src.stacey_nz), d(src.stacey_weight)
        s.st_rvp, s.st_rvs = d(src.stacey_rho_vp), d(src.stacey_rho_vs)
        s.nsrc = len(src.source_ispec)
        s.src_ispec = i(src.source_ispec)
        s.sourcearrays = d(src.sourcearrays)
        s.stf = d(src.stf)
        s.nstep_total = src.stf.shape[1] if s.nsrc else 0
        s.nstage = nstage
        s.nrec = len(src.rec_ispec)
        s.rec_ispec = i(src.rec_ispec)
        s.hxir, s.hgammar = d(src.hxir), d(src.hgammar)
        s.cosrot, s.sinrot = float(src.cosrot), float(src.sinrot)
        s.seismotype = int(getattr(src, "seismotype", 1) if seismotype is None else seismotype)
        s.deltat, s.deltatover2, s.deltatsquareover2 = dt, dto2, dt2o2
        an = getattr(src, "aniso", None)
        if an is not None:
            s.ispec_is_anisotropic = i(an["ispec"])
            s.c11, s.c13, s.c15 = d(an["c11"]), d(an["c13"]), d(an["c15"])
            s.c33, s.c35, s.c55 = d(an["c33"]), d(an["c35"]), d(an["c55"])
        s.time_scheme = int(src.time_scheme)
        s.alpha_lddrk, s.beta_lddrk = d(ALPHA_LDDRK), d(BETA_LDDRK)
        at = getattr(src, "atten", None)
        if at is not None:
            s.att_a1, s.att_b1, s.att_a2, s.att_b2 = d(at["a1"]), d(at["b1"]), d(at["a2"]), d(at["b2"])
            s.att_itau1, s.att_phi1 = d(at["itau1"]), d(at["phi1"])
            s.att_itau2, s.att_phi2 = d(at["itau2"]), d(at["phi2"])
        ac = getattr(src, "acoustic", None)
        if ac is not None:
            s.ispec_is_acoustic = i(ac["ispec"])
            s.rmass_inverse_acoustic = d(ac["rmass"])
            s.nstacey_ac = len(ac["st_iglob"])
            s.st_ac_iglob, s.st_ac_w, s.st_ac_rvp = i(ac["st_iglob"]), d(ac["st_w"]), d(ac["st_rvp"])
            s.nfree_ac = len(ac["free_iglob"])
            s.free_ac_iglob = i(ac["free_iglob"])
            s.ncpl_ac = len(ac["cpl_ac_iglob"])
            s.cpl_ac_iglob = i(ac["cpl_ac_iglob"])
            s.cpl_ac_nx, s.cpl_ac_nz, s.cpl_ac_w = d(ac["cpl_ac_nx"]), d(ac["cpl_ac_nz"]), d(ac["cpl_ac_w"])
            s.ncpl_el = len(ac["cpl_el_iglob"])
            s.cpl_el_iglob = i(ac["cpl_el_iglob"])
            s.cpl_el_nx, s.cpl_el_nz, s.cpl_el_w = d(ac["cpl_el_nx"]), d(ac["cpl_el_nz"]), d(ac["cpl_el_w"])
            s.use_trick = int(bool(ac.get("use_trick", False)))
            if "cpl_ac_elpt" in ac:
                s.cpl_ac_elpt, s.cpl_el_acpt = i(ac["cpl_ac_elpt"]), i(ac["cpl_el_acpt"])
        s.DT = float(src.dt)
        pm = getattr(src, "pml", None)
        if pm is not None:
            s.pml_region = i(pm["region"])
            s.pml_K_x, s.pml_K_z = d(pm["K_x"]), d(pm["K_z"])
            s.pml_d_x, s.pml_d_z = d(pm["d_x"]), d(pm["d_z"])
            s.pml_alpha_x, s.pml_alpha_z = d(pm["alpha_x"]), d(pm["alpha_z"])
            s.npml_bnd_el, s.pml_bnd_el = len(pm["bnd_el"]), i(pm["bnd_el"])
            s.npml_bnd_ac, s.pml_bnd_ac = len(pm["bnd_ac"]), i(pm["bnd_ac"])
            if "visco" in pm and at is not None and np.any(pm["visco"]):
                s.pml_visco = i(pm["visco"])
                s.att_teps1, s.att_teps2 = d(at["teps1"]), d(at["teps2"])
                s.att_mu1, s.att_mu2 = d(at["mu1"]), d(at["mu2"])
        if adj_src is not None:
            s.adj_src = d(adj_src)
            s.nstep_total = int(np.asarray(adj_src).shape[1])
        self._keep = keep
        self.s = s
        self.h = lib().sf2d_oracle_create(ctypes.byref(s), precision)
        if not self.h:
            raise RuntimeError("oracle creation failed")
        self.dtype = np.float32 if precision == 4 else np.float64
        self.it = 0

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            lib().sf2d_oracle_destroy(h)
            self.h = None

    def _size(self, which):
        if which in (HESS1, HESS2, RHO_AC_KL, KAPPA_AC_KL):
            return (self.s.nspec, 5, 5)
        if which >= POT:
            return (self.s.nglob,)
        if which <= VELOC_LDDRK:
            return (self.s.nglob, 2)
        if which >= RHO_KL:
            return (self.s.nspec, 5, 5)
        return (self.s.nspec, 5, 5, 3)

    def accumulate_kernels(self, b_displ):
        b = np.ascontiguousarray(b_displ, dtype=self.dtype).reshape(self.s.nglob, 2)
        if lib().sf2d_oracle_accumulate_kernels(self.h, b.ctypes.data) != 0:
            raise RuntimeError("kernel accumulation failed")

    def accumulate_kernels_acoustic(self, b_pot):
        b = np.ascontiguousarray(b_pot, dtype=self.dtype).reshape(self.s.nglob)
        if lib().sf2d_oracle_accumulate_kernels_acoustic(self.h, b.ctypes.data) != 0:
            raise RuntimeError("fluid kernel accumulation failed")

    def accumulate_hessian(self, b_accel):
        b = np.ascontiguousarray(b_accel, dtype=self.dtype).reshape(self.s.nglob, 2)
        if lib().sf2d_oracle_accumulate_hessian(self.h, b.ctypes.data) != 0:
            raise RuntimeError("Hessian accumulation failed")

    def get(self, which):
        out = np.empty(self._size(which), dtype=self.dtype)
        if lib().sf2d_oracle_get(self.h, which, out.ctypes.data) != 0:
            raise RuntimeError(f"oracle field {which} unavailable")
        return out

    def set(self, which, arr):
        arr = np.ascontiguousarray(arr, dtype=self.dtype).reshape(self._size(which))
        if lib().sf2d_oracle_set(self.h, which, arr.ctypes.data) != 0:
            raise RuntimeError(f"oracle field {which} unavailable")

    @property
    def displ(self):
        return self.get(DISPL)

    @property
    def veloc(self):
        return self.get(VELOC)

    @property
    def accel(self):
        return self.get(ACCEL)

    def run(self, nstep: int, nthreads: int = 0) -> np.ndarray:
        """Advance nstep time steps; return seismograms (nrec, nstep, 2) float64."""
        seis = np.zeros((self.s.nrec, nstep, 2), dtype=np.float64)
        rc = lib().sf2d_oracle_run(self.h, nstep, seis.ctypes.data_as(_dp), nthreads)
        if rc != 0:
            raise RuntimeError(f"oracle failed with status {rc}")
        self.it += nstep
        return seis


def checkpoint_fields(o):
    """Fields that define the state of a Newmark run (for segment checkpointing)."""
    names = [DISPL, VELOC, ACCEL]
    if o.db.atten is not None:
        names += [E1, E11, E13, ATT_OLD]
    if getattr(o.db, "acoustic", None) is not None:
        names += [POT, POT_DOT, POT_DOT_DOT]
    return {k: o.get(k) for k in names}


def kernels(db, adj_src, checkpoint_every=200, precision=4, nthreads=0, hessian=False):
    """Forward run from rest with a state checkpoint every `checkpoint_every`
    steps, then, segment by segment in reverse, the forward segment is
    recomputed from its checkpoint (frames of the displacement and, with fluid
    elements, of the potential kept) and the adjoint field, driven by
    `adj_src` (nrec, nstep, 2) in time order, or by `adj_src(synthetics)` when
    it is a function, is advanced over it; adjoint step it is paired with
    forward step NSTEP - it + 1 (src/specfem2D/iterate_time_undoatt.F90:193-601).

    Returns a dict: ``seis`` and ``adj_seis`` (nrec, nstep, 2); the solid
    kernels ``rho``, ``kappa``, ``mu`` scaled as save_adjoint_kernels.f90:134-141
    does (zero in fluid elements); with fluid elements ``rho_ac`` and
    ``kappa_ac`` (compute_kernels.f90:420-436, deltat included, zero in solid
    elements); with `hessian` the approximate Hessian ``hess1``, ``hess2``."""
    nstep = db.nstep
    fluid = getattr(db, "acoustic", None) is not None
    fwd = Oracle(db, precision)
    ckpts = {}
    seis = np.zeros((db.rec_ispec.size, nstep, 2))
    for s0 in range(0, nstep, checkpoint_every):
        ckpts[s0] = checkpoint_fields(fwd)
        n = min(checkpoint_every, nstep - s0)
        seis[:, s0:s0 + n] = fwd.run(n, nthreads)
    if callable(adj_src):
        adj_src = adj_src(seis)
    adj = Oracle(db, precision, adj_src=adj_src)
    adj_seis = np.zeros_like(seis)
    done = 0
    for s0 in sorted(ckpts, reverse=True):
        n = min(checkpoint_every, nstep - s0)
        rec = Oracle(db, precision)
        for k, v in ckpts[s0].items():
            rec.set(k, v)
        rec.it = s0
        _set_step(rec, s0)
        frames, pframes, aframes = [], [], []
        for _ in range(n):
            rec.run(1, nthreads)
            frames.append(rec.displ)
            if fluid:
                pframes.append(rec.get(POT))
            if hessian:
                aframes.append(rec.accel)
        for k in range(n - 1, -1, -1):
            adj_seis[:, done:done + 1] = adj.run(1, nthreads)
            done += 1
            adj.accumulate_kernels(frames[k])
            if fluid:
                adj.accumulate_kernels_acoustic(pframes[k])
            if hessian:
                adj.accumulate_hessian(aframes[k])
    f = np.float32 if precision == 4 else np.float64
    dtf = f(db.deltat) if precision == 4 else float(db.dt)
    out = {"seis": seis, "adj_seis": adj_seis,
           "rho": (-db.rhostore.astype(f) * dtf) * adj.get(RHO_KL),
           "mu": (-f(2.0) * db.mustore.astype(f) * dtf) * adj.get(MU_KL),
           "kappa": (-db.kappastore.astype(f) * dtf) * adj.get(KAPPA_KL)}
    if fluid:
        out["rho_ac"] = adj.get(RHO_AC_KL)
        out["kappa_ac"] = adj.get(KAPPA_AC_KL)
    if hessian:
        out["hess1"], out["hess2"] = adj.get(HESS1), adj.get(HESS2)
    return out


def adjoint_kernels(db, adj_src, checkpoint_every=200, precision=4, nthreads=0, hessian=False):
    """The solid part of `kernels` as a tuple: (synthetics, adjoint traces,
    rho_kl, kappa_kl, mu_kl), then hess1, hess2 with `hessian`."""
    k = kernels(db, adj_src, checkpoint_every, precision, nthreads, hessian)
    t = (k["seis"], k["adj_seis"], k["rho"], k["kappa"], k["mu"])
    return t + (k["hess1"], k["hess2"]) if hessian else t


def gradient(db, observed, checkpoint_every=200, precision=4, nthreads=0):
    """Misfit, synthetics and sensitivity kernels of the L2 waveform misfit
    chi = 1/2 sum_r sum_it |s - d|^2 dt, with the adjoint source s - d
    (the run of adjoint_kernels).  Returns (chi, synthetics, rho_kl,
    kappa_kl, mu_kl)."""
    misfit = {}

    def residual(syn):
        resid = syn - observed
        misfit["chi"] = 0.5 * float(np.sum(resid ** 2)) * float(db.dt)
        return resid

    seis, _, rho_kl, kappa_kl, mu_kl = adjoint_kernels(db, residual, checkpoint_every, precision, nthreads)
    return misfit["chi"], seis, rho_kl, kappa_kl, mu_kl


def _set_step(o, it):
    """Moves the state's step counter (source time functions are indexed by it)."""
    lib().sf2d_oracle_set_step(o.h, it)


def smooth(db, fields, sigma_h: float, sigma_v: float) -> np.ndarray:
    """smooth_sem's CPU smoothing of per-element-point fields (nfields, nspec, 5, 5)
    on the Database's mesh, float32 (all pairs: small meshes only)."""
    fl = np.ascontiguousarray(np.asarray(fields, dtype=np.float32).reshape(-1, db.nspec, 5, 5))
    x = np.ascontiguousarray(db.coord[db.ibool, 0], dtype=np.float32)
    z = np.ascontiguousarray(db.coord[db.ibool, 1], dtype=np.float32)
    jac = np.ascontiguousarray(db.jacobian, dtype=np.float32)
    w = db.gll.wgll_dble
    wsq = np.ascontiguousarray((w[None, :] * w[:, None]).astype(np.float32))  # [j][i] = w_i w_j
    ib = np.ascontiguousarray(db.ibool, dtype=np.int32)
    out = np.zeros_like(fl)
    f = lib().sf2d_oracle_smooth
    f.restype = ctypes.c_int
    rc = f(db.nspec, db.nglob, ib.ctypes.data_as(_ip), x.ctypes.data_as(ctypes.c_void_p),
           z.ctypes.data_as(ctypes.c_void_p), jac.ctypes.data_as(ctypes.c_void_p), wsq.ctypes.data_as(ctypes.c_void_p),
           fl.shape[0], fl.ctypes.data_as(ctypes.c_void_p), ctypes.c_float(sigma_h), ctypes.c_float(sigma_v),
           out.ctypes.data_as(ctypes.c_void_p))
    if rc != 0:
        raise RuntimeError("oracle smoothing failed")
    return out


def max_threads() -> int:
    return int(lib().sf2d_oracle_max_threads())
