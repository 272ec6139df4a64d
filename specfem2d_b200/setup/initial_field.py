"""Analytical initial wavefields (Par_file ``initialfield = .true.``).

Restates the mode branch (source_type 6 of the first SOURCE entry) of
src/specfem2D/prepare_initial_field.F90:

* the wave speed is taken at one point, ``cploc = rho_vpstore / rhostore`` of
  the first GLL point of the first element, in CUSTOM_REAL (:210-211);
* mode (n, m) = (2, 3) of a rectangular membrane with amplitude 1 (:312-326),
  angular frequency ``omega = cploc sqrt((n pi / Lx)^2 + (m pi / Lz)^2)`` with
  Lx, Lz the extent of the mesh coordinates (:398);
* at every global point, with x, z scaled to [0, 1] over the mesh extent and
  t = -t0 (the time offset of :375):
  ``y = sin(n pi x) sin(m pi z) cos(omega t)``,
  ``y' = -omega sin(n pi x) sin(m pi z) sin(omega t)``, ``y'' = -omega^2 y``
  (:548-558), in double, stored in CUSTOM_REAL;
* an elastic medium moves in z only, a fluid takes y as its potential chi
  (:559-571).

With an initial field no source is injected
(compute_forces_viscoelastic_calling_routine.F90:90,
compute_forces_viscoacoustic_calling_routine.F90:143) and the first LDDRK
stage takes the ordinary update (update_displacement_LDDRK.F90:70,103).
The plane-wave branches (source types 1-5) need the Bielak boundary
conditions and are not restated.
"""
from __future__ import annotations

import math

import numpy as np

PI = 3.141592653589793
MODE_N, MODE_M, MODE_A = 2, 3, 1.0


def mode_omega(cploc: float, xmin: float, xmax: float, zmin: float, zmax: float) -> float:
    """Angular frequency of the (2, 3) membrane mode (prepare_initial_field.F90:398)."""
    return cploc * math.sqrt((MODE_N * PI / (xmax - xmin)) ** 2 + (MODE_M * PI / (zmax - zmin)) ** 2)


def initial_mode_field(coord: np.ndarray, rho_vpstore: np.ndarray, rhostore: np.ndarray, t0: float,
                       acoustic: bool) -> dict:
    """Initial field of the membrane mode at time -t0.

    ``coord`` (nglob, 2) float64; ``rho_vpstore``, ``rhostore`` the CUSTOM_REAL
    material stores (nspec, 5, 5).  Returns float32 arrays: ``pot``, ``pot_dot``,
    ``pot_dot_dot`` (nglob,) for a fluid, or ``displ``, ``veloc``, ``accel``
    (nglob, 2) for a solid, and the mode's ``omega``."""
    cploc = float(np.float32(np.float32(rho_vpstore.flat[0]) / np.float32(rhostore.flat[0])))
    x_all, z_all = coord[:, 0], coord[:, 1]
    xmin, xmax = float(x_all.min()), float(x_all.max())
    zmin, zmax = float(z_all.min()), float(z_all.max())
    om = mode_omega(cploc, xmin, xmax, zmin, zmax)
    t = 0.0 - t0
    x = (x_all - xmin) / (xmax - xmin)
    z = (z_all - zmin) / (zmax - zmin)
    s1, s2 = np.sin(MODE_N * PI * x), np.sin(MODE_M * PI * z)
    # left-to-right products, as the Fortran expressions evaluate
    y = ((MODE_A * s1) * s2) * math.cos(om * t)
    ydot = (((-om * MODE_A) * s1) * s2) * math.sin(om * t)
    ydd = -(om * om) * y
    if acoustic:
        return dict(pot=y.astype(np.float32), pot_dot=ydot.astype(np.float32), pot_dot_dot=ydd.astype(np.float32),
                    omega=om)
    z0 = np.zeros_like(y)
    return dict(displ=np.stack([z0, y], axis=1).astype(np.float32),
                veloc=np.stack([z0, ydot], axis=1).astype(np.float32),
                accel=np.stack([z0, ydd], axis=1).astype(np.float32), omega=om)
