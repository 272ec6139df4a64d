"""Synthetic workloads with the shapes of the benchmark configurations.

No public dataset is involved: meshes come from the internal mesher
(flat or sinusoidal top interface), materials from seeded analytic laws.

* ``c1_homogeneous``: 4000 m x 3000 m, 80 x 60 quads, vp 3000, vs 1732,
  rho 2700, free top, Stacey elsewhere, vertical force 500 m below the
  surface at x = 2000 m, Ricker 10 Hz, dt 1e-3, 20 surface receivers.
* ``c2_geometry``: 20 km x 8 km, 800 x 320 quads, vp rising linearly
  2000 -> 4500 m/s with depth below a 1 km top layer, vs = vp / 1.73,
  Gardner rho = 310 vp^0.25, 5 % Gaussian random perturbation (correlation
  length 200 m, seed 2), Ricker 8 Hz source, dt 5e-4, 400 receivers.  With
  ``elastic_only`` the 1 km top layer is elastic (vp 2000) and the sides and
  bottom use Stacey instead of CPML.
"""
from __future__ import annotations

import numpy as np

from .setup.gll import NGLL
from .setup.mesh import internal_mesh
from .setup.solver_setup import Source, build_database


def _gll_points(mesh, gll):
    from .setup.mesh import _interp_nodes, _shape_tables

    sh, _, _ = _shape_tables(gll, mesh.ngnod)
    return _interp_nodes(mesh, sh)


def gaussian_random_field(xmax, zmax, corr_len, seed, spacing=None):
    """Zero-mean, unit-std isotropic Gaussian random field on a regular grid.

    White noise filtered in the wavenumber domain by exp(-k^2 L^2 / 4), i.e.
    a Gaussian correlation of length L.  Returns (grid x, grid z, values).
    """
    h = spacing or corr_len / 4.0
    nxg = int(np.ceil(xmax / h)) + 1
    nzg = int(np.ceil(zmax / h)) + 1
    rng = np.random.default_rng(seed)
    w = rng.standard_normal((nzg, nxg))
    kx = 2 * np.pi * np.fft.fftfreq(nxg, d=h)
    kz = 2 * np.pi * np.fft.fftfreq(nzg, d=h)
    k2 = kz[:, None] ** 2 + kx[None, :] ** 2
    f = np.real(np.fft.ifft2(np.fft.fft2(w) * np.exp(-k2 * corr_len ** 2 / 4.0)))
    f = (f - f.mean()) / f.std()
    return np.arange(nxg) * h, np.arange(nzg) * h, f


def _bilinear(gx, gz, f, x, z):
    h = gx[1] - gx[0]
    ix = np.clip((x / h).astype(np.int64), 0, len(gx) - 2)
    iz = np.clip((z / h).astype(np.int64), 0, len(gz) - 2)
    tx = np.clip(x / h - ix, 0.0, 1.0)
    tz = np.clip(z / h - iz, 0.0, 1.0)
    return ((1 - tx) * (1 - tz) * f[iz, ix] + tx * (1 - tz) * f[iz, ix + 1]
            + (1 - tx) * tz * f[iz + 1, ix] + tx * tz * f[iz + 1, ix + 1])


def c1_homogeneous(nstep: int = 2000, nrec: int = 20):
    xmax, zmax, nx, nz = 4000.0, 3000.0, 80, 60
    interfaces = [([0.0, xmax], [0.0, 0.0]), ([0.0, xmax], [zmax, zmax])]
    mesh = internal_mesh(0.0, xmax, nx, interfaces, [nz], absorb=(True, True, False, True))
    src = Source(x=2000.0, z=zmax - 500.0, source_type=1, time_function_type=1, f0=10.0,
                 anglesource_deg=0.0, factor=1.0e10)
    xs = np.linspace(200.0, 3800.0, nrec)
    recs = [(float(x), zmax) for x in xs]
    return build_database(mesh, 2700.0, 3000.0, 1732.0, [src], recs, nstep, 1.0e-3,
                          stacey=True, external_model=False)


def c2_geometry(nstep: int = 6000, nrec: int = 400, elastic_only: bool = True, scale: int = 1):
    """The 800 x 320 coupled-model geometry (``scale`` divides the element counts)."""
    if not elastic_only:
        raise NotImplementedError("acoustic layer of the coupled model")
    xmax, zmax = 20000.0, 8000.0
    nx, nz = 800 // scale, 320 // scale
    interfaces = [([0.0, xmax], [0.0, 0.0]), ([0.0, xmax], [zmax, zmax])]
    mesh = internal_mesh(0.0, xmax, nx, interfaces, [nz], absorb=(True, True, False, True))
    from .setup.gll import GLL

    gll = GLL()
    x, z = _gll_points(mesh, gll)
    depth = zmax - z
    seafloor = 1000.0
    vp = np.where(depth <= seafloor, 2000.0,
                  2000.0 + 2500.0 * np.clip((depth - seafloor) / (zmax - seafloor), 0.0, 1.0))
    gx, gz, f = gaussian_random_field(xmax, zmax, 200.0, seed=2)
    vp = vp * (1.0 + 0.05 * _bilinear(gx, gz, f, x, z))
    vs = vp / 1.73
    rho = 310.0 * vp ** 0.25
    src = Source(x=10000.0, z=zmax - 500.0, source_type=1, time_function_type=1, f0=8.0,
                 anglesource_deg=0.0, factor=1.0e10)
    xs = np.linspace(100.0, xmax - 100.0, nrec)
    recs = [(float(xr), zmax - 10.0) for xr in xs]
    return build_database(mesh, rho, vp, vs, [src], recs, nstep, 5.0e-4, stacey=True,
                          external_model=True)


def algorithmic_bytes_elastic(nspec: int, nglob: int) -> int:
    """Bytes of one fused elastic isotropic Newmark step in the reference data
    layout: 25 points x (xix, xiz, gammax, gammaz, kappa, mu, ibool) x 4 B per
    element, and u, v, a read + write plus rmass_x, rmass_z read per point."""
    return 700 * nspec + 56 * nglob
