"""Host side of a kernel (SIMULATION_TYPE = 3) run: adjoint sources and the
kernels derived from rho_kl, kappa_kl, mu_kl.

* ``cross_correlation_adjoint_source`` restates the reference's adjoint-source
  tool, src/auxiliaries/adj_seismogram.f90: a Welch window over
  [tstart, tend] (index rule floor/ceiling of :270-290, taper of :330-335),
  centred-difference velocity and acceleration of the trace (:345-360), the
  normalisation N = dt sum(w s a) and the source w v / N (:362-370), written
  only for the selected component (1 = X, 3 = Z, 4 = X and Z; :372-385).
  The result is what the solver reads from SEM/*.adj; read_adj_source
  (compute_arrays_source.f90:166-300) stores it in CUSTOM_REAL.
* ``derived_kernels`` restates the second half of save_kernels_elastic
  (save_adjoint_kernels.f90:159-169): rho' = rho + kappa + mu kernels,
  beta = 2 (mu - 4/3 mu/kappa kappa), alpha = 2 (1 + 4/3 mu/kappa) kappa,
  bulk_c = 2 kappa, bulk_beta = 2 mu, in CUSTOM_REAL.
"""
from __future__ import annotations

import math

import numpy as np

f32 = np.float32


def cross_correlation_adjoint_source(t: np.ndarray, traces: np.ndarray, tstart: float, tend: float,
                                     adj_comp: int):
    """Adjoint source of a cross-correlation traveltime measurement.

    ``t`` (nstep,) sample times and ``traces`` (nstep, 2) the X and Z
    displacement traces as the solver wrote them; returns (adj, norms) with
    adj (nstep, 2) float64 (X, Z) and norms = {"X": N_x, "Z": N_z}, where
    a norm below 1e-40 in magnitude zeroes that component."""
    nstep = len(t)
    t0 = float(t[0])
    deltat = (float(t[-1]) - t0) / float(nstep - 1)
    istart = math.floor((tstart - t0) / deltat) + 1
    iend = math.ceil((tend - t0) / deltat) + 1
    if istart < 1:
        istart = 1
    if istart > nstep:
        istart = nstep - 1
    if iend < istart:
        iend = istart + 1
    if iend > nstep:
        iend = nstep
    if istart >= iend:
        raise ValueError("empty time window")
    it = np.arange(1, nstep + 1, dtype=np.float64)
    win = np.zeros(nstep)
    sel = (it >= istart) & (it <= iend)
    win[sel] = 1.0 - (2 * (it[sel] - istart) / (iend - istart) - 1.0) ** 2
    adj = np.zeros((nstep, 2))
    norms = {}
    for c, name, comp_id in ((0, "X", 1), (1, "Z", 3)):
        s = np.asarray(traces[:, c], dtype=np.float64)
        v = np.zeros(nstep)
        v[1:-1] = (s[2:] - s[:-2]) / (2 * deltat)
        v[0] = (s[1] - s[0]) / deltat
        v[-1] = (s[-1] - s[-2]) / deltat
        a = np.zeros(nstep)
        a[1:-1] = (v[2:] - v[:-2]) / (2 * deltat)
        a[0] = (v[1] - v[0]) / deltat
        a[-1] = (v[-1] - v[-2]) / deltat
        # Fortran's sum(): one left-to-right pass
        nn = 0.0
        for k in range(nstep):
            nn += win[k] * s[k] * a[k]
        nn = deltat * nn
        norms[name] = nn
        ft = v * win / nn if abs(nn) > 1e-40 else np.zeros(nstep)
        if comp_id == adj_comp or adj_comp == 4:
            adj[:, c] = ft
    return adj, norms


def derived_kernels(rho_kl, kappa_kl, mu_kl, rhostore, kappastore, mustore) -> dict:
    """rho', alpha, beta, bulk_c and bulk_beta kernels from the primary ones (float32)."""
    rk, kk, mk = (np.asarray(a, dtype=f32) for a in (rho_kl, kappa_kl, mu_kl))
    mul, kappal = np.asarray(mustore, dtype=f32), np.asarray(kappastore, dtype=f32)
    four_thirds = f32(4.0 / 3.0)
    ratio = four_thirds * mul / kappal
    return dict(rhop=rk + kk + mk,
                beta=f32(2.0) * (mk - ratio * kk),
                alpha=f32(2.0) * (f32(1.0) + ratio) * kk,
                bulk_c=f32(2.0) * kk,
                bulk_beta=f32(2.0) * mk)
