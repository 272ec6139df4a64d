"""Autotuner for the tile-staged kernels: elements per tile x threads per CTA.

Each candidate builds its tiling, runs a few warm-up steps, then times
`steps` single launches with CUDA events (sf2d_time_kernels) and keeps the
configuration with the smallest time per step (element kernel plus
shared-point kernel).  Candidates whose shared memory does not fit are
skipped.

    python -m specfem2d_b200.autotune --workload c2_geometry
"""
from __future__ import annotations

import argparse
import json
import time

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
