"""A small elastic inversion case shared by the gradient tests (CPU and GPU).

2-D medium 4 km x 2.4 km (40 x 24 quads), vp 3000 m/s rising 0.3 /s with
depth, vs = vp / 1.73, rho 2500; true model = a +5 % rho / +10 % kappa, mu
Gaussian anomaly (radius 300 m); one Ricker 8 Hz force at 30 degrees,
9 surface receivers, 900 Newmark steps of 1.5 ms, Stacey on three sides.
"""
from __future__ import annotations

import numpy as np

from specfem2d_b200.configs import _gll_points
from specfem2d_b200.setup.gll import GLL
from specfem2d_b200.setup.mesh import internal_mesh
from specfem2d_b200.setup.solver_setup import Source, build_database

NX, NZ, L, H = 40, 24, 4000.0, 2400.0


class Case:
    def __init__(self, nstep: int = 900, qmu: float | None = None):
        interfaces = [([0.0, L], [0.0, 0.0]), ([0.0, L], [H, H])]
        self.mesh = internal_mesh(0.0, L, NX, interfaces, [NZ], absorb=(True, True, False, True))
        self.x, self.z = _gll_points(self.mesh, GLL())
        self.nstep = nstep
        self.qmu = qmu
        vp0 = 3000.0 + 0.3 * (H - self.z)
        vs0 = vp0 / 1.73
        self.rho0 = 2500.0 + 0 * self.x
        self.mu0 = self.rho0 * vs0 ** 2
        self.kappa0 = self.rho0 * vp0 ** 2 - self.mu0

    def db(self, rho, kappa, mu):
        vp = np.sqrt((kappa + mu) / rho)
        vs = np.sqrt(mu / rho)
        src = Source(x=1200.0, z=H - 600.0, source_type=1, time_function_type=1, f0=8.0,
                     anglesource_deg=30.0, factor=1e10)
        recs = [(float(xr), H) for xr in np.linspace(400, 3600, 9)]
        q = {}
        if self.qmu is not None:
            q = dict(qkappa=np.full_like(rho, 9999.0), qmu=np.full_like(rho, self.qmu))
        return build_database(self.mesh, rho, vp, vs, [src], recs, self.nstep, 1.5e-3, stacey=True,
                              external_model=True, **q)

    def anomaly(self, cx=2400.0, cz=1200.0, r=300.0):
        return np.exp(-((self.x - cx) ** 2 + (self.z - cz) ** 2) / r ** 2)

    def true_db(self):
        a = self.anomaly()
        return self.db(self.rho0 * (1 + 0.05 * a), self.kappa0 * (1 + 0.1 * a), self.mu0 * (1 + 0.1 * a))

    def start_db(self):
        return self.db(self.rho0, self.kappa0, self.mu0)
