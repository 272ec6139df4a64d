"""Reader for the subset of DATA/Par_file, DATA/SOURCE and DATA/STATIONS on the hot path.

Follows the reference's ``key = value`` convention with ``#`` comments
(src/shared/param_reader.c:98-160, src/shared/read_parameter_file.F90) and the
material / region tables that follow ``nbmodels`` and ``nbregions``
(src/shared/read_material_table.f90, src/meshfem2D/read_regions.f90).
Fortran literals such as ``2.0d-2`` and ``.true.`` are converted.
"""
from __future__ import annotations

import math
import re


def _fvalue(tok: str):
    t = tok.strip()
    tl = t.lower()
    if tl in (".true.", "true", "t"):
        return True
    if tl in (".false.", "false", "f"):
        return False
    try:
        return int(t)
    except ValueError:
        pass
    try:
        return float(re.sub(r"[dD]", "e", t))
    except ValueError:
        return t


def read_par_file(path: str) -> dict:
    """Return {key: value}, plus ``materials`` (list of token lists), ``regions``
    and ``receiver_sets`` (one dict per ``nrec`` block, read_parameter_file.F90
    reads nreceiversets blocks of nrec, xdeb, zdeb, xfin, zfin,
    record_at_surface_same_vertical)."""
    out: dict = {"materials": [], "regions": [], "receiver_sets": []}
    rec_keys = ("nrec", "xdeb", "zdeb", "xfin", "zfin", "record_at_surface_same_vertical")
    with open(path) as f:
        lines = [ln.split("#", 1)[0].rstrip() for ln in f]
    lines = [ln for ln in lines if ln.strip()]
    i = 0
    while i < len(lines):
        ln = lines[i]
        if "=" in ln:
            key, val = ln.split("=", 1)
            key = key.strip()
            out[key] = _fvalue(val)
            if key == "nrec":
                out["receiver_sets"].append({})
            if key in rec_keys and out["receiver_sets"]:
                out["receiver_sets"][-1][key] = out[key]
            if key == "nbmodels":
                n = int(out[key])
                out["materials"] = [lines[i + 1 + k].split() for k in range(n)]
                i += n
            elif key == "nbregions":
                n = int(out[key])
                out["regions"] = [[int(v) for v in lines[i + 1 + k].split()[:5]] for k in range(n)]
                i += n
        i += 1
    return out


def read_source_file(path: str) -> list:
    """Return a list of dicts, one per source block (read_source_file.f90)."""
    sources = []
    cur = None
    with open(path) as f:
        for ln in f:
            s = ln.split("#", 1)[0].strip()
            if not s or "=" not in s:
                continue
            k, v = s.split("=", 1)
            k = k.strip()
            if k == "source_surf":
                cur = {}
                sources.append(cur)
            if cur is None:
                cur = {}
                sources.append(cur)
            cur[k] = _fvalue(v)
    return sources


def read_stations(path: str) -> list:
    """STATIONS lines: station network x z elevation burial."""
    st = []
    with open(path) as f:
        for ln in f:
            p = ln.split()
            if len(p) >= 4:
                st.append((p[0], p[1], float(p[2]), float(p[3])))
    return st


def material_from_row(row) -> dict:
    """Material table row (read_materials.f90:116-215).

    Isotropic ``n 1 rho vp vs 0 0 Qkappa Qmu ...``; anisotropic
    ``n 2 rho c11 c13 c15 c33 c35 c55 c12 c23 c25 c22 Qkappa Qmu``, whose
    cp = sqrt(c33/rho) and cs = sqrt(c55/rho) feed the isotropic stores used
    by the mass matrix and Stacey.
    """
    vals = [_fvalue(v) for v in row]
    kind = int(vals[1])
    if kind == -1:
        # tomographic material: values come from TOMOGRAPHY_FILE (read_materials.f90:192-205)
        return dict(index=int(vals[0]), kind=-1, rho=0.0, vp=0.0, vs=0.0, qkappa=9999.0, qmu=9999.0)
    if kind == 2:
        rho = float(vals[2])
        c = [float(v) for v in vals[3:9]]
        qk = float(vals[13]) if len(vals) > 13 and float(vals[13]) > 0.1 else 9999.0
        qm = float(vals[14]) if len(vals) > 14 and float(vals[14]) > 0.1 else 9999.0
        return dict(index=int(vals[0]), kind=2, rho=rho, vp=math.sqrt(c[3] / rho), vs=math.sqrt(c[5] / rho),
                    qkappa=qk, qmu=qm, c11=c[0], c13=c[1], c15=c[2], c33=c[3], c35=c[4], c55=c[5])
    return dict(index=int(vals[0]), kind=kind, rho=float(vals[2]), vp=float(vals[3]),
                vs=float(vals[4]), qkappa=float(vals[7]), qmu=float(vals[8]))
