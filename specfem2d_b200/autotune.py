"""Autotuner for the tile-staged kernels and for packed batches.

* ``autotune_elastic``: elements per tile x threads per CTA of a solid mesh.
  Each candidate builds its tiling, runs a few warm-up steps, then times
  `steps` single launches with CUDA events (sf2d_time_kernels) and keeps the
  configuration with the smallest time per step (element kernel plus
  shared-point kernel).  Candidates whose shared memory does not fit are
  skipped.
* ``autotune_coupled``: fluid tile size and the solid CPML tiles' size and
  threads of a coupled mesh.  The solid and fluid kernels overlap on two
  streams, so each candidate is timed on whole graph-queued steps.
* ``autotune_batch``: members per packed mesh of a gradient batch (shots or
  models per launch), timed on whole gradients of a sample of the members.

    python -m specfem2d_b200.autotune --workload c2_geometry
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

DEFAULT_TILES = (32, 48, 64, 96, 128)
DEFAULT_THREADS = (128, 256, 512)


def autotune_elastic(db, tiles=DEFAULT_TILES, threads=DEFAULT_THREADS, steps: int = 20, warmup: int = 5,
                     verbose: bool = False):
    """Returns (best (tile_elems, threads), list of result dicts)."""
    from .runtime import ElasticSolver, SF2DError

    results = []
    for te in tiles:
        for nt in threads:
            try:
                sol = ElasticSolver(db, tile_elems=te, threads_per_block=nt)
            except SF2DError as e:
                results.append({"tile_elems": te, "threads": nt, "error": str(e)})
                continue
            try:
                sol.enqueue(warmup)
                sol.synchronize(120)
                ms = sol.time_kernels(steps)
                info = sol.layout_info()
            finally:
                sol.close()
            r = {"tile_elems": te, "threads": nt, "tile_ms": ms[0], "shared_ms": ms[1], "step_ms": ms[2],
                 "ntiles": info["ntiles"], "nshared": info["nshared"], "smem_bytes": info["smem_bytes"]}
            results.append(r)
            if verbose:
                print(json.dumps(r), flush=True)
    ok = [r for r in results if "step_ms" in r]
    if not ok:
        raise RuntimeError("no autotune candidate ran")
    best = min(ok, key=lambda r: r["step_ms"])
    return (best["tile_elems"], best["threads"]), results


def _time_steps(sol, steps: int, warmup: int) -> float:
    """Milliseconds per step of graph-queued steps (host clock around a synchronised run)."""
    sol.prepare()
    sol.enqueue(warmup)
    sol.synchronize(120)
    t0 = time.perf_counter()
    sol.enqueue(steps)
    sol.synchronize(120)
    return (time.perf_counter() - t0) * 1e3 / steps


def autotune_coupled(db, tile_elems: int = 32, threads: int = 256, fluid_tiles=(32, 64),
                     pml=((16, 128), (32, 256)), steps: int = 64, warmup: int = 8, verbose: bool = False):
    """Returns (best (fluid_tile_elems, pml_tile_elems, pml_threads), results) for a coupled Database."""
    from .coupled import CoupledSolver
    from .runtime import SF2DError

    results = []
    for ft in fluid_tiles:
        for pt, pn in pml:
            try:
                sol = CoupledSolver(db, tile_elems=tile_elems, threads_per_block=threads, fluid_tile_elems=ft,
                                    pml_tile_elems=pt, pml_threads_per_block=pn)
            except SF2DError as e:
                results.append({"fluid_tile_elems": ft, "pml_tile_elems": pt, "pml_threads": pn, "error": str(e)})
                continue
            try:
                ms = _time_steps(sol, steps, warmup)
            finally:
                sol.close()
            r = {"fluid_tile_elems": ft, "pml_tile_elems": pt, "pml_threads": pn, "step_ms": ms}
            results.append(r)
            if verbose:
                print(json.dumps(r), flush=True)
    ok = [r for r in results if "step_ms" in r]
    if not ok:
        raise RuntimeError("no autotune candidate ran")
    best = min(ok, key=lambda r: r["step_ms"])
    return (best["fluid_tile_elems"], best["pml_tile_elems"], best["pml_threads"]), results


def autotune_batch(members, observed, sizes=(1, 2, 4, 8), checkpoint_every: int = 100, sample: int = 8,
                   verbose: bool = False):
    """Members per packed mesh for gradient batches: times whole gradients of
    the first `sample` members packed `size` at a time and returns (best
    size, results) with the seconds per member of each size."""
    from . import batch
    from .fwi import FWIGradient

    sample_m = list(members[:sample])
    sample_o = list(observed[:sample])
    results = []
    for size in sizes:
        if size > len(sample_m):
            continue
        t = 0.0
        for b0 in range(0, len(sample_m), size):
            grp = sample_m[b0:b0 + size]
            db, _ = batch.pack(grp) if len(grp) > 1 else (grp[0], None)
            obs = np.concatenate(sample_o[b0:b0 + size], axis=0)
            g = FWIGradient(db, checkpoint_every)
            t0 = time.perf_counter()
            seis = g.forward()
            g.backward(seis - obs)
            t += time.perf_counter() - t0
            g.close()
        r = {"members_per_batch": size, "s_per_member": t / len(sample_m)}
        results.append(r)
        if verbose:
            print(json.dumps(r), flush=True)
    best = min(results, key=lambda r: r["s_per_member"])
    return best["members_per_batch"], results


def main():
    import os
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench  # workload construction shared with the benchmark

    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="c2_geometry")
    ap.add_argument("--steps", type=int, default=20)
    args = ap.parse_args()
    t0 = time.time()
    db = bench.build_workload(args.workload, 256)
    best, _ = autotune_elastic(db, steps=args.steps, verbose=True)
    print(json.dumps({"best_tile_elems": best[0], "best_threads": best[1], "seconds": time.time() - t0}))


if __name__ == "__main__":
    main()
