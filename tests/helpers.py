"""Shared helpers for the test suite (fixture loading, error metrics)."""
from __future__ import annotations

import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_golden(name):
    with open(os.path.join(GOLDEN, name + ".json")) as f:
        cfg = json.load(f)
    seis = dict(np.load(os.path.join(GOLDEN, name + "_seis.npz")))
    mesh = os.path.join(GOLDEN, name + "_mesh.npz")
    if os.path.exists(mesh):
        cfg["external_mesh"] = dict(np.load(mesh))
    return cfg, seis


def load_kernel_golden(name):
    """(config, adjoint arrays, kernel-run log values) of a kernel example
    without REF_SEIS (tests/golden/make_golden.py KERNEL_ONLY)."""
    with open(os.path.join(GOLDEN, name + ".json")) as f:
        cfg = json.load(f)
    ref = dict(np.load(os.path.join(GOLDEN, name + "_adjoint.npz")))
    with open(os.path.join(GOLDEN, name + "_adjoint.json")) as f:
        log = json.load(f)
    return cfg, ref, log


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def initial_mode_run(db, precision):
    """Oracle traces (nstep, 2) of a run started from the Database's analytical
    initial potential (the initial_mode_LDDRK example)."""
    import oracle

    o = oracle.Oracle(db, precision)
    f = db.initial_field
    o.set(oracle.POT, f["pot"])
    o.set(oracle.POT_DOT, f["pot_dot"])
    o.set(oracle.POT_DOT_DOT, f["pot_dot_dot"])
    return o.run(db.nstep)[0]


def within_fp32_band(x, center, o32, o64):
    """`x` (nstep, 2) is as close to `center` as the FP32 oracle is to the FP64
    oracle (relative L2 at most 1.5x theirs), on the first 100, 1000 and all
    steps, per component."""
    return all(rel_l2(x[:n, c], center[:n, c]) <= 1.5 * rel_l2(o32[:n, c], o64[:n, c])
               for n in (100, 1000, x.shape[0]) for c in (0, 1))
