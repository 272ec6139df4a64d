"""Tomographic (gridded) velocity models: TOMOGRAPHY_FILE of the Par_file.

Restates define_external_model_from_tomo_file.f90: the file layout read by
read_tomo_file (:536-831; four header lines, then x z vp vs rho [qp qs]
records scanning x fastest) and the bilinear ``interpolate`` with its edge
and corner rules (:146-335) and ``searchInf`` (:66-144).  GLL points of the
tomographic material take the interpolated values at their global
coordinates (:386-470); other materials keep their table values.
"""
from __future__ import annotations

import numpy as np

TINYVAL = 1.0e-9


def read_tomo_file(path):
    """Return (x (nx,), z (nz,), vp (nx, nz), vs, rho), all float64."""
    with open(path) as f:
        lines = [ln.split("#", 1)[0].strip() for ln in f]
    lines = [ln for ln in lines if ln]
    nx, nz = (int(v) for v in lines[2].split()[:2])
    rec = np.array([[float(v) for v in ln.split()[:5]] for ln in lines[4:4 + nx * nz]])
    x = rec[:nx, 0].copy()
    z = rec[::nx, 1].copy()
    vp = rec[:, 2].reshape(nz, nx).T.copy()
    vs = rec[:, 3].reshape(nz, nx).T.copy()
    rho = rec[:, 4].reshape(nz, nx).T.copy()
    return x, z, vp, vs, rho


def search_inf(arr, value, d=1.0e-9):
    """1-based index of the grid cell holding ``value`` (searchInf)."""
    n = len(arr)
    if n == 1:
        return 1
    if value < arr[0]:
        return 1
    if value >= arr[n - 1]:
        return n - 1
    k = 1
    while arr[k - 1] < value:
        k += 1
    return k - 1 if abs(arr[k - 1] - value) > d else k


def interpolate(xa, ya, f, x, y):
    """Bilinear interpolation of f (len(xa), len(ya)) at (x, y) with the
    reference's branch order for points on or beyond the grid edges."""
    nx, ny = len(xa), len(ya)
    minx, maxx, miny, maxy = xa.min(), xa.max(), ya.min(), ya.max()

    def le(a, b):   # a < b or |a - b| < TINYVAL
        return a < b or abs(a - b) < TINYVAL

    def ge(a, b):
        return a > b or abs(a - b) < TINYVAL

    def xcell(v):
        i = search_inf(xa, v)
        return (i, xa[i - 1], xa[i]) if i < nx else (i, xa[i - 2], xa[i - 1])

    def ycell(v):
        j = search_inf(ya, v)
        return (j, ya[j - 1], ya[j]) if j < ny else (j, ya[j - 2], ya[j - 1])

    F = lambda i, j: f[i - 1, j - 1]  # noqa: E731  (1-based access)
    if le(x, minx) and le(y, miny):
        return F(1, 1)
    if x > maxx and ge(y, maxy):
        return F(nx, ny)
    if le(x, minx) and ge(y, maxy):
        return F(1, ny)
    if ge(x, maxx) and le(y, miny):
        return F(nx, 1)
    if ge(x, minx) and le(x, maxx) and le(y, miny):
        y1, y2 = ya[0], ya[1]
        i, x1, x2 = xcell(x)
        denom = (x2 - x1) * (y2 - y1)
        return (F(i, 1) * (x2 - x) * (y2 - y1) + F(i + 1, 1) * (x - x1) * (y2 - y1)) / denom
    if ge(x, minx) and le(x, maxx) and ge(y, maxy):
        y1, y2 = ya[ny - 2], ya[ny - 1]
        i, x1, x2 = xcell(x)
        j = ny - 1
        denom = (x2 - x1) * (y2 - y1)
        return (F(i, j + 1) * (x2 - x) * (y2 - y1) + F(i + 1, j + 1) * (x - x1) * (y2 - y1)) / denom
    if le(x, minx) and ge(y, miny) and le(y, maxy):
        x1, x2 = xa[0], xa[1]
        j, y1, y2 = ycell(y)
        denom = (x2 - x1) * (y2 - y1)
        return (F(1, j) * (x2 - x1) * (y2 - y) + F(1, j + 1) * (x2 - x1) * (y - y1)) / denom
    if ge(x, maxx) and ge(y, miny) and le(y, maxy):
        x1, x2 = xa[nx - 2], xa[nx - 1]
        i = nx - 1
        j, y1, y2 = ycell(y)
        denom = (x2 - x1) * (y2 - y1)
        return (F(i + 1, j) * (x2 - x1) * (y2 - y) + F(i + 1, j + 1) * (x2 - x1) * (y - y1)) / denom
    i, x1, x2 = xcell(x)
    j, y1, y2 = ycell(y)
    denom = (x2 - x1) * (y2 - y1)
    return (F(i, j) * (x2 - x) * (y2 - y) + F(i + 1, j) * (x - x1) * (y2 - y)
            + F(i, j + 1) * (x2 - x) * (y - y1) + F(i + 1, j + 1) * (x - x1) * (y - y1)) / denom


def tomo_values(tomo, coord, ibool, elements):
    """(rho, vp, vs) at every GLL point of ``elements`` (float32 values, as the
    CUSTOM_REAL rhoext/vpext/vsext arrays hold them).  Returns three arrays of
    shape (len(elements), 5, 5)."""
    x, z, vp, vs, rho = tomo
    cache = {}
    out = np.zeros((3, len(elements)) + ibool.shape[1:], dtype=np.float32)
    for k, e in enumerate(elements):
        for j in range(ibool.shape[1]):
            for i in range(ibool.shape[2]):
                g = int(ibool[e, j, i])
                v = cache.get(g)
                if v is None:
                    xm, zm = float(coord[g, 0]), float(coord[g, 1])
                    v = (interpolate(x, z, rho, xm, zm), interpolate(x, z, vp, xm, zm),
                         interpolate(x, z, vs, xm, zm))
                    cache[g] = v
                out[:, k, j, i] = v
    return out[0], out[1], out[2]
