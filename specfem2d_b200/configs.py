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


def c2_coupled(nstep: int = 6000, nrec: int = 400, scale: int = 1, rec_depth: float = 50.0,
               time_scheme: int = 1, use_trick: bool = False, pml_thickness: int = 0):
    """Coupled fluid-solid model: 20 km x 8 km, 800 x 320 quads (``scale``
    divides both counts), a 1 km water layer (vp 1500 m/s, rho 1020 kg/m^3,
    vs 0) over rock with vp rising linearly 2000 -> 4500 m/s from the sea
    floor to the bottom, vs = vp / 1.73, Gardner rho = 310 vp^0.25, and a 5 %
    Gaussian random perturbation (correlation 200 m, seed 2) of the rock; free
    sea surface, absorbing sides and bottom (Stacey, or CPML layers of
    ``pml_thickness`` elements); pressure source 500 m deep in the water,
    Ricker 8 Hz; ``nrec`` pressure receivers ``rec_depth`` below the sea
    surface; dt 5e-4 s (Courant ~0.55 at the fastest rock)."""
    xmax, zmax = 20000.0, 8000.0
    nx, nz = 800 // scale, 320 // scale
    interfaces = [([0.0, xmax], [0.0, 0.0]), ([0.0, xmax], [zmax, zmax])]
    mesh = internal_mesh(0.0, xmax, nx, interfaces, [nz], absorb=(True, True, False, True))
    from .setup.gll import GLL

    x, z = _gll_points(mesh, GLL())
    depth = zmax - z
    seafloor = 1000.0
    water = (zmax - z.mean(axis=(1, 2))) < seafloor  # whole elements: the sea floor is an element boundary
    vp = 2000.0 + 2500.0 * np.clip((depth - seafloor) / (zmax - seafloor), 0.0, 1.0)
    gx, gz, f = gaussian_random_field(xmax, zmax, 200.0, seed=2)
    vp = vp * (1.0 + 0.05 * _bilinear(gx, gz, f, x, z))
    vs = vp / 1.73
    rho = 310.0 * vp ** 0.25
    vp[water], vs[water], rho[water] = 1500.0, 0.0, 1020.0
    src = Source(x=10000.0, z=zmax - 500.0, source_type=1, time_function_type=1, f0=8.0,
                 anglesource_deg=0.0, factor=1.0e10)
    xs = np.linspace(100.0, xmax - 100.0, nrec)
    recs = [(float(xr), zmax - rec_depth) for xr in xs]
    pml = dict(nelem_thickness=pml_thickness) if pml_thickness > 0 else None
    return build_database(mesh, rho, vp, vs, [src], recs, nstep, 5.0e-4, stacey=pml is None,
                          external_model=True, time_scheme=time_scheme, seismotype=4, use_trick=use_trick,
                          **({"pml": pml} if pml else {}))


def algorithmic_bytes_coupled(nspec_el: int, nglob_el: int, nspec_ac: int, nglob_ac: int,
                              npml_el: int = 0, npml_ac: int = 0) -> int:
    """Bytes of one coupled Newmark step in the reference layout: the solid
    step over its elements and points plus, per fluid element, 25 points x
    (xix, xiz, gammax, gammaz, rho, ibool) x 4 B and, per fluid point, chi,
    chi_dot, chi_dot_dot read + write and rmass read.  Each CPML element adds,
    per GLL point, its six damping profiles (K, d, alpha in x and z, 48 B in
    double) and rho J or J / kappa (4 B), and its memory variables read +
    write: 12 floats in the solid (strain 8, displacement 4: 96 B), 6 in the
    fluid (48 B)."""
    return (700 * nspec_el + 56 * nglob_el + 600 * nspec_ac + 28 * nglob_ac
            + 25 * (48 + 4 + 96) * npml_el + 25 * (48 + 4 + 48) * npml_ac)


def c2_geometry(nstep: int = 6000, nrec: int = 400, elastic_only: bool = True, scale: int = 1):
    """The 800 x 320 model geometry with rock everywhere (``scale`` divides the element counts);
    ``elastic_only=False`` gives the coupled model of c2_coupled."""
    if not elastic_only:
        return c2_coupled(nstep=nstep, nrec=nrec, scale=scale)
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


def c4_gradient(nstep: int = 4000, nrec: int = 200, true_model: bool = False, qmu=None, scale: int = 1,
                shot_x: float = 12500.0, dt: float | None = None):
    """Elastic 1000 x 400 quads over 25 km x 10 km (``scale`` divides both
    counts).  Background: vp = 2500 m/s + 0.2 /s x depth, vs = vp / 1.73,
    Gardner rho; the true model adds two +-10 % Gaussian anomalies (radius
    1 km, centres 3-7 km deep drawn with seed 4).  One Ricker 8 Hz vertical
    force 500 m deep, 200 surface receivers, Stacey on three sides.  dt
    defaults to 4e-4 x scale (Courant ~0.46 with the smallest GLL spacing at
    every scale).  At full scale 4000 steps (1.6 s) end before any wave has
    travelled to the anomalies and back, so the misfit of that run is zero to
    rounding; at quarter scale the same step count covers 6.4 s."""
    dt = 4.0e-4 * scale if dt is None else dt
    xmax, zmax = 25000.0, 10000.0
    nx, nz = 1000 // scale, 400 // scale
    interfaces = [([0.0, xmax], [0.0, 0.0]), ([0.0, xmax], [zmax, zmax])]
    mesh = internal_mesh(0.0, xmax, nx, interfaces, [nz], absorb=(True, True, False, True))
    from .setup.gll import GLL

    x, z = _gll_points(mesh, GLL())
    depth = zmax - z
    vp = 2500.0 + 0.2 * depth
    if true_model:
        rng = np.random.default_rng(4)
        for sign in (1.0, -1.0):
            cx = rng.uniform(6000.0, 19000.0)
            cz = rng.uniform(3000.0, 7000.0)
            vp = vp * (1.0 + sign * 0.10 * np.exp(-((x - cx) ** 2 + (z - cz) ** 2) / 1000.0 ** 2))
    vs = vp / 1.73
    rho = 310.0 * vp ** 0.25
    src = Source(x=shot_x, z=zmax - 500.0, source_type=1, time_function_type=1, f0=8.0, anglesource_deg=0.0,
                 factor=1.0e10)
    xs = np.linspace(250.0, xmax - 250.0, nrec)
    recs = [(float(xr), zmax) for xr in xs]
    q = {}
    if qmu is not None:
        q = dict(qkappa=np.full_like(vp, 9999.0), qmu=np.full_like(vp, float(qmu)))
    return build_database(mesh, rho, vp, vs, [src], recs, nstep, dt, stacey=True, external_model=True, **q)


def random_layered_model(seed: int, nx: int, nz: int, nstep: int, dx: float = 25.0, dt: float = 4.0e-4,
                         nrec: int = 20):
    """A random layered elastic model (3 to 6 flat layers, vp 2000..4500 m/s,
    vs = vp / 1.73, Gardner rho) of nx x nz quads of dx metres, one Ricker
    8 Hz force and `nrec` surface receivers."""
    rng = np.random.default_rng(seed)
    xmax, zmax = nx * dx, nz * dx
    interfaces = [([0.0, xmax], [0.0, 0.0]), ([0.0, xmax], [zmax, zmax])]
    mesh = internal_mesh(0.0, xmax, nx, interfaces, [nz], absorb=(True, True, False, True))
    from .setup.gll import GLL

    x, z = _gll_points(mesh, GLL())
    nl = int(rng.integers(3, 7))
    tops = np.sort(rng.uniform(0.0, zmax, nl - 1))
    vps = np.sort(rng.uniform(2000.0, 4500.0, nl))[::-1]  # faster at depth
    layer = np.searchsorted(tops, z)
    vp = vps[np.clip(layer, 0, nl - 1)]
    vs = vp / 1.73
    rho = 310.0 * vp ** 0.25
    src = Source(x=float(rng.uniform(0.2, 0.8) * xmax), z=zmax - 10.0 * dx, source_type=1,
                 time_function_type=1, f0=8.0, anglesource_deg=0.0, factor=1.0e10)
    recs = [(float(xr), zmax) for xr in np.linspace(0.05 * xmax, 0.95 * xmax, nrec)]
    return build_database(mesh, rho, vp, vs, [src], recs, nstep, dt, stacey=True, external_model=True)


def c5_model_sizes(count: int = 48, seed: int = 6, lo=(100, 50), hi=(1200, 500)):
    """Uneven mesh sizes (nx, nz) drawn with `seed` between lo and hi (aspect 2:1 kept)."""
    rng = np.random.default_rng(seed)
    f = rng.uniform(0.0, 1.0, count)
    nx = (lo[0] + f * (hi[0] - lo[0])).astype(int)
    nz = np.maximum(lo[1], (nx * (hi[1] / hi[0])).astype(int))
    return list(zip(nx.tolist(), nz.tolist()))


def c3_viscoelastic(nstep: int = 8000, time_scheme: int = 1, scale: int = 1, nrec: int = 100):
    """1600 x 800 quads over 40 km x 20 km under a sinusoidal surface (amplitude
    200 m, wavelength 5 km); vp rising smoothly 2500 -> 6000 m/s with depth,
    vs = vp / 1.73, Gardner rho; 3 SLS with Qkappa 200, Qmu 60; moment-tensor
    source (Mxx, Mzz, Mxz drawn with seed 3) 2 km deep, Ricker 5 Hz;
    dt 3e-4 (Courant ~0.42 at 6000 m/s with 25 m elements); Newmark
    (time_scheme 1) or LDDRK (2)."""
    import math

    xmax, zmax = 40000.0, 20000.0
    nx, nz = 1600 // scale, 800 // scale
    interfaces = [([0.0, xmax], [0.0, 0.0]), ([0.0, xmax], [zmax, zmax])]

    def topo(x):
        return zmax + 200.0 * math.sin(2.0 * math.pi * x / 5000.0)

    mesh = internal_mesh(0.0, xmax, nx, interfaces, [nz], absorb=(True, True, False, True), topography_fn=topo)
    from .setup.gll import GLL

    x, z = _gll_points(mesh, GLL())
    depth = np.clip(zmax - z, 0.0, zmax)
    vp = 2500.0 + 3500.0 * (depth / zmax) ** 0.8
    vs = vp / 1.73
    rho = 310.0 * vp ** 0.25
    rng = np.random.default_rng(3)
    mxx, mzz, mxz = rng.uniform(-1.0, 1.0, 3)
    src = Source(x=20000.0, z=zmax - 2000.0, source_type=2, time_function_type=1, f0=5.0,
                 Mxx=float(mxx), Mzz=float(mzz), Mxz=float(mxz), factor=1.0e10)
    xs = np.linspace(500.0, xmax - 500.0, nrec)
    recs = [(float(xr), topo(float(xr))) for xr in xs]
    return build_database(mesh, rho, vp, vs, [src], recs, nstep, 3.0e-4, stacey=True, external_model=True,
                          time_scheme=time_scheme, qkappa=np.full_like(vp, 200.0), qmu=np.full_like(vp, 60.0))


def algorithmic_bytes_viscoelastic(nspec: int, nglob: int, time_scheme: int = 1) -> int:
    """Bytes of one viscoelastic 3-SLS step in the reference layout: the elastic
    step plus, per element GLL point, e1 e11 e13 (3 SLS) read + write (72 B),
    the A/B coefficients (48 B) and the three previous strains read + write
    (24 B) for Newmark; LDDRK does 6 stages, each with the element data, the
    memory variables and their LDDRK copies read + write (144 B), 1/tau and
    phi (48 B) per element point and u, v, u_L, v_L read + write, a written
    and rmass read per global point (88 B)."""
    if time_scheme == 1:
        return 700 * nspec + 56 * nglob + 3600 * nspec
    return 6 * (nspec * (700 + 25 * 192) + nglob * 88)
