"""Misfit gradients through the C ABI's forward/backward pair (sf2d_fwi_*).

`FWIGradient` wraps one medium + source: `forward()` runs the elastic
Newmark time loop from rest on the GPU, saving a state checkpoint every
`checkpoint_every` steps, and returns the receiver traces; `backward(adj)`
runs the adjoint sweep (forward segments recomputed from their checkpoints)
and returns the scaled sensitivity kernels rho_kl, kappa_kl, mu_kl in the
reference layout, exactly as SPECFEM2D defines them (relative-perturbation
kernels; mu_kl is the derivative at fixed lambda + 2/3 mu, the convention of
compute_kernels.f90).

`l2_misfit_gradient` is the L2 waveform misfit chi = 1/2 sum |s - d|^2 dt with
adjoint source s - d.  `SeismogramOperator` is a thin torch.autograd.Function
test binding: model log-perturbations -> seismograms, with the gradient of any
scalar loss obtained from one adjoint sweep.
"""
from __future__ import annotations

import ctypes

import numpy as np

from .runtime import _check, _d, _f, build_desc, load_library


class FWIGradient:
    def __init__(self, db, checkpoint_every: int = 200, tile_elems: int = 32, threads_per_block: int = 256,
                 hessian: bool = False):
        """`hessian` also accumulates the approximate Hessian (see hessian())."""
        if int(db.time_scheme) != 1:
            raise ValueError("the gradient is implemented for the Newmark scheme")
        lib = load_library()
        d, keep = build_desc(db, tile_elems, 1, threads_per_block)
        rho = np.ascontiguousarray(db.rhostore, dtype=np.float32)
        kap = np.ascontiguousarray(db.kappastore, dtype=np.float32)
        h = ctypes.c_void_p()
        _check(lib.sf2d_fwi_create(ctypes.byref(d), rho.ctypes.data_as(_f), kap.ctypes.data_as(_f),
                                   int(checkpoint_every), ctypes.byref(h)))
        self._h, self._lib = h, lib
        if hessian:
            _check(lib.sf2d_fwi_enable_hessian(h))
        self.nrec, self.nstep, self.nspec = len(db.rec_ispec), db.nstep, db.nspec
        self.dt = float(db.dt)
        del keep

    def close(self):
        if getattr(self, "_h", None):
            self._lib.sf2d_fwi_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def forward(self) -> np.ndarray:
        seis = np.zeros((self.nrec, self.nstep, 2), dtype=np.float64)
        _check(self._lib.sf2d_fwi_forward(self._h, seis.ctypes.data_as(_d)))
        return seis

    def backward(self, adj_src):
        adj = np.ascontiguousarray(np.asarray(adj_src, dtype=np.float32).reshape(self.nrec, self.nstep, 2))
        out = [np.zeros((self.nspec, 5, 5), dtype=np.float32) for _ in range(3)]
        _check(self._lib.sf2d_fwi_backward(self._h, adj.ctypes.data_as(_f), *[o.ctypes.data_as(_f) for o in out]))
        return tuple(out)

    def hessian(self):
        """rhorho_el_Hessian_final1 and _final2 (nspec, 5, 5) of the last backward():
        the time integrals of |b_accel|^2 and of accel_adj . b_accel
        (compute_kernels.f90:749-800)."""
        out = [np.zeros((self.nspec, 5, 5), dtype=np.float32) for _ in range(2)]
        _check(self._lib.sf2d_fwi_hessian(self._h, out[0].ctypes.data_as(_f), out[1].ctypes.data_as(_f)))
        return tuple(out)

    def adjoint_seismograms(self) -> np.ndarray:
        """Receiver traces (nrec, nstep, 2) of the adjoint field of the last backward()."""
        seis = np.zeros((self.nrec, self.nstep, 2), dtype=np.float64)
        _check(self._lib.sf2d_fwi_adjoint_seismograms(self._h, seis.ctypes.data_as(_d)))
        return seis


def l2_misfit_gradient(db, observed, checkpoint_every: int = 200, **kw):
    """(chi, synthetics, rho_kl, kappa_kl, mu_kl) for chi = 1/2 sum_r sum_it |s - d|^2 dt."""
    g = FWIGradient(db, checkpoint_every, **kw)
    seis = g.forward()
    resid = seis - observed
    chi = 0.5 * float(np.sum(resid ** 2)) * float(db.dt)
    kernels = g.backward(resid)
    g.close()
    return (chi, seis) + kernels


def quadrature_weights(db) -> np.ndarray:
    """w_i w_j J at every element GLL point: turns kernels into gradients of a sum over points."""
    w = db.gll.wgll_dble
    return (w[None, :] * w[:, None])[None] * db.jacobian.astype(np.float64)


def SeismogramOperator():
    """torch.autograd.Function: (dln_rho, dln_kappa, dln_mu, builder) -> seismograms.

    `builder(rho, kappa, mu)` returns a Database for the perturbed model; the
    backward pass turns dLoss/dseismograms g into the adjoint source g / dt and
    returns w J K for each parameter (the gradient of the loss with respect to
    the log-perturbation at each element GLL point).
    """
    import torch

    class _Op(torch.autograd.Function):
        @staticmethod
        def forward(ctx, dln_rho, dln_kappa, dln_mu, base, builder, checkpoint_every):
            rho0, kap0, mu0 = base
            rho = rho0 * np.exp(dln_rho.detach().cpu().numpy())
            kap = kap0 * np.exp(dln_kappa.detach().cpu().numpy())
            mu = mu0 * np.exp(dln_mu.detach().cpu().numpy())
            db = builder(rho, kap, mu)
            g = FWIGradient(db, checkpoint_every)
            seis = g.forward()
            ctx.g, ctx.wj, ctx.dt = g, quadrature_weights(db), float(db.dt)
            return torch.from_numpy(seis)

        @staticmethod
        def backward(ctx, grad_seis):
            adj = grad_seis.detach().cpu().numpy() / ctx.dt
            rk, kk, mk = ctx.g.backward(adj)
            ctx.g.close()
            wj = ctx.wj
            out = [torch.from_numpy(wj * k.astype(np.float64)) for k in (rk, kk, mk)]
            return out[0], out[1], out[2], None, None, None

    return _Op


def summed_shot_gradient(shots, observed, checkpoint_every: int = 200, batch_size: int = 0, gradient_fn=None):
    """Misfit and kernels summed over the shots of one model: the gradient of
    sum_s chi_s, as a survey inversion needs it.

    `shots` are Databases of the same mesh and model that differ in their
    sources (batch.shots_on_model); `observed` the data of each shot.  The
    shots are split over the ranks of the process group (one GPU each), each
    rank runs its share packed `batch_size` at a time (0 = all in one packed
    mesh) and sums its kernels, and one all-reduce adds the ranks' sums (NCCL
    on GPUs, gloo on CPU).  `gradient_fn(db, observed) -> (chi, synthetics,
    rho_kl, kappa_kl, mu_kl)` defaults to l2_misfit_gradient.  Returns
    (chi, rho_kl, kappa_kl, mu_kl), the kernels as float64 (nspec, 5, 5)."""
    from . import batch
    from .distributed import rank_world, shard, sum_over_ranks

    if gradient_fn is None:
        def gradient_fn(db, obs):
            return l2_misfit_gradient(db, obs, checkpoint_every=checkpoint_every)
    rank, world = rank_world()
    mine = shard([s.nspec for s in shots], rank, world)
    nspec = shots[0].nspec
    acc = np.zeros((4, nspec, 5, 5), dtype=np.float64)  # chi in acc[0, 0, 0, 0]
    size = batch_size if batch_size > 0 else max(1, len(mine))
    for b0 in range(0, len(mine), size):
        grp = [shots[k] for k in mine[b0:b0 + size]]
        obs = [observed[k] for k in mine[b0:b0 + size]]
        if len(grp) == 1:
            chi, _, *kern = gradient_fn(grp[0], obs[0])
            parts = [[k] for k in kern]
        else:
            packed, idx = batch.pack(grp)
            chi, _, *kern = gradient_fn(packed, np.concatenate(obs, axis=0))
            parts = [batch.split_elements(k, idx) for k in kern]
        acc[0, 0, 0, 0] += chi
        for c in range(3):
            for p in parts[c]:
                acc[1 + c] += p
    total = sum_over_ranks(acc)
    return float(total[0, 0, 0, 0]), total[1], total[2], total[3]
