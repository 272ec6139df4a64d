"""Benchmark of the SPECFEM2D time-marching hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload c2_coupled|c2_geometry|c1|...] [--tile-elems T]

A "step" is one Newmark time step of the whole mesh.  The metric is GLL
point-updates per second (global points x steps / s).  With N > 1 (torchrun,
one process per GPU) every rank advances its own replica of the workload (the
shots of a survey are independent), so scaling is weak and `value` sums all
ranks' point-updates over the slowest rank's time.

`--impl reference` times the CPU restatement of the reference solver (the
oracle; the Fortran xspecfem2D cannot be built without a Fortran compiler)
on all host cores, on the same workload, over a bounded number of steps.

Prints one JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import copy
import json
import math
import os
import pickle
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CACHE = os.path.join("/tmp", "sf2d_bench_cache")


def _make_workload(name: str, nstep: int, scale: int = 1):
    from specfem2d_b200 import configs

    if scale != 1 and name not in ("c2_coupled", "c2_coupled_stacey", "c2_geometry", "c3_viscoelastic",
                                   "c3_viscoelastic_lddrk"):
        raise SystemExit(f"--scale applies to the c2 and c3 workloads, not {name}")
    if name == "c2_coupled":
        return configs.c2_coupled(nstep=nstep, pml_thickness=20 // scale, scale=scale)
    if name == "c2_coupled_stacey":
        return configs.c2_coupled(nstep=nstep, scale=scale)
    if name == "c2_geometry":
        return configs.c2_geometry(nstep=nstep, scale=scale)
    if name == "c1":
        return configs.c1_homogeneous(nstep=nstep)
    if name == "c4_elastic":
        return configs.c4_gradient(nstep=nstep)
    if name == "c3_viscoelastic":
        return configs.c3_viscoelastic(nstep=nstep, time_scheme=1, scale=scale)
    if name == "c3_viscoelastic_lddrk":
        return configs.c3_viscoelastic(nstep=nstep, time_scheme=2, scale=scale)
    raise SystemExit(f"unknown workload {name}")


def build_workload(name: str, nstep: int, rank: int = 0, dist=None, scale: int = 1):
    """The workload's Database (``scale`` divides the element counts: profiling
    cases).  With several ranks, rank 0 builds it and the others load its
    pickle (one set-up's memory instead of one per rank)."""
    if dist is None:
        return _make_workload(name, nstep, scale)
    os.makedirs(CACHE, exist_ok=True)
    path = os.path.join(CACHE, f"{name}_{nstep}_{scale}.pkl")
    if rank == 0:
        db = _make_workload(name, nstep, scale)
        with open(path + ".tmp", "wb") as f:
            pickle.dump(db, f, protocol=5)
        os.replace(path + ".tmp", path)
    dist.barrier()
    if rank != 0:
        with open(path, "rb") as f:
            db = pickle.load(f)
    return db


# steps of the configuration's whole run (the end-to-end leg over the full run)
WORKLOAD_NSTEP = {"c1": 2000, "c2_coupled": 6000, "c3_viscoelastic": 8000}


# DRAM bytes one step's solid tile launches move (read + write), measured with
# ncu on one B200 for the workload and tile configuration of the key
# (workload, tile elements, threads, fluid tile elements, CPML tile elements,
# CPML threads); the roofline's "traffic" reports it beside the algorithmic bytes
TILE_TRAFFIC = {
    ("c2_coupled", 32, 256, 64, 16, 128): 233.0e6 + 43.45e6 + 71.07e6 + 0.40e6 + 1.25e6,
    # 376.16 MB per launch on the quarter-scale model (80,000 elements), x16 elements
    ("c3_viscoelastic", 32, 256, 64, 16, 128): 376.16e6 * 16,
    # 64-element tiles (the autotuner's choice): 371.10 MB per launch at quarter scale, x16
    ("c3_viscoelastic", 64, 256, 64, 16, 128): 371.10e6 * 16,
    # 48-element tiles (the autotuner's choice with the 64-register bound): 369.33 MB at quarter scale, x16
    ("c3_viscoelastic", 48, 256, 64, 16, 128): 369.33e6 * 16,
}
TRAFFIC_SOURCE = {
    ("c2_coupled", 32, 256, 64, 16, 128): "ncu dram__bytes_read.sum + dram__bytes_write.sum of one step's solid "
                                          "tile launches (early, late and CPML tiles), one capture",
    ("c3_viscoelastic", 32, 256, 64, 16, 128): "ncu dram__bytes_read.sum + dram__bytes_write.sum of one tile "
                                               "launch on the quarter-scale model (--scale 4), scaled by the "
                                               "element count (x16)",
    ("c3_viscoelastic", 64, 256, 64, 16, 128): "ncu dram__bytes_read.sum + dram__bytes_write.sum of one tile "
                                               "launch (64-element tiles) on the quarter-scale model (--scale 4), "
                                               "mean of two launches, scaled by the element count (x16)",
    ("c3_viscoelastic", 48, 256, 64, 16, 128): "ncu dram__bytes_read.sum + dram__bytes_write.sum of one tile "
                                               "launch (48-element tiles, 64 registers) on the quarter-scale model "
                                               "(--scale 4), mean of two launches, scaled by the element count (x16)",
}

WORKLOAD_DESC = {
    "c2_coupled": ("800x320-element (20 km x 8 km, 4,100,481 GLL points) coupled fluid-solid model: 1 km "
                   "water layer (vp 1500, rho 1020, 32,000 acoustic elements) over rock with vp 2000->4500 "
                   "with depth, vs=vp/1.73, Gardner rho, 5% Gaussian random field (corr. 200 m, seed 2); "
                   "20-element CPML on the sides and bottom (28,000 layer elements, 1,600 of them fluid); "
                   "pressure source 500 m deep, Ricker 8 Hz, dt 5e-4, 400 pressure receivers"),
    "c2_coupled_stacey": ("the c2_coupled model with Stacey conditions on the sides and bottom instead of "
                          "the CPML layers"),
    "c2_geometry": ("800x320-element (20 km x 8 km, 4,100,481 GLL points) mesh of the coupled "
                    "acoustic-elastic configuration, run elastic-only: the 1 km top layer is elastic "
                    "(vp 2000) and Stacey replaces the 20-element CPML; vp 2000->4500 with depth, "
                    "vs=vp/1.73, Gardner rho, 5% Gaussian random field (corr. 200 m, seed 2), "
                    "Ricker 8 Hz force, dt 5e-4, 400 receivers"),
    "c1": "80x60 homogeneous elastic, Stacey L/R/B, free top, Ricker 10 Hz, 20 receivers",
    "c4_elastic": ("forward run of the 1000x400-element (25 km x 10 km, 6,405,601 GLL points) isotropic "
                   "starting model of the gradient configuration: linear-gradient background, Stacey "
                   "sides and bottom, Ricker 8 Hz, 200 receivers, dt 4e-4"),
    "c3_viscoelastic": ("1600x800-element (40 km x 20 km, 20,489,601 GLL points) viscoelastic model under "
                        "sinusoidal topography (200 m, 5 km), 3 SLS Qkappa 200 Qmu 60, vp 2500-6000, "
                        "seeded moment tensor, Ricker 5 Hz, dt 3e-4, Newmark"),
    "c3_viscoelastic_lddrk": "the same viscoelastic model advanced with the 6-stage LDDRK scheme",
}


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", str(self.gpu)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
            return
        # nvidia-smi's start-up (NVML initialisation) must not overlap the timed
        # region: wait for its first two samples
        t0 = time.time()
        while len(self.lines) < 2 and time.time() - t0 < 15.0 and self.proc.poll() is None:
            time.sleep(0.02)

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax.append(float(p[2]))
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def time_oracle(db, max_steps: int, target_s: float = 15.0, nthreads: int = 0):
    """Times the CPU oracle (FP32) on a bounded number of steps; returns (steps, seconds, threads)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle  # noqa: E402  (CPU baseline leg only)

    o = oracle.Oracle(db, 4)
    t0 = time.perf_counter()
    o.run(2, nthreads=nthreads)
    t_step = (time.perf_counter() - t0) / 2
    n = int(max(2, min(max_steps, math.ceil(target_s / max(t_step, 1e-6)))))
    t0 = time.perf_counter()
    o.run(n, nthreads=nthreads)
    dt = time.perf_counter() - t0
    threads = nthreads if nthreads > 0 else oracle.max_threads()
    return n, dt, threads


def run_reference_fwi(args, rank):
    """The CPU restatement's gradient (forward, checkpointed reverse sweep) on
    the smallest model of the FWI workload, per shot."""
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle  # noqa: E402  (reference arm only)

    if args.workload == "c4_fwi_shots":
        from specfem2d_b200 import configs

        # one shot of the same model at 1/8 of the element count per direction (bounded CPU sample)
        db = configs.c4_gradient(nstep=args.fwi_steps, scale=8)
        nglobs = [(4 * 1000 + 1) * (4 * 400 + 1)] * args.models
    else:
        models = fwi_members(args.models, args.fwi_steps, args.fwi_set)
        db = min(models, key=lambda m: m.nspec)
        nglobs = [m.nglob for m in models]
    t0 = time.perf_counter()
    oracle.gradient(db, np.zeros((len(db.rec_ispec), db.nstep, 2)), checkpoint_every=100, precision=4)
    t_sample = time.perf_counter() - t0
    # per shot of the workload: the sample's time scaled by the mean point count
    scale = float(np.mean(nglobs)) / float(db.nglob)
    dt = t_sample * scale
    threads = oracle.max_threads()
    line = {"metric": "s per FWI gradient per shot", "value": dt, "unit": "s", "impl": "reference",
            "n_gpus": args.gpus, "steps": args.fwi_steps, "warmup": 0, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": args.workload, "description": FWI_WORKLOADS[args.workload],
                       "model_set": args.fwi_set, "models": len(nglobs), "sample_nspec": db.nspec,
                       "sample_seconds": t_sample},
            "cpu_baseline": {"value": dt, "unit": "s", "cores": threads, "kind": "port",
                             "sample": f"one gradient of a {db.nspec}-element model ("
                                       f"{db.nstep} steps, {t_sample:.1f} s) scaled by the mean point count "
                                       f"of the {len(nglobs)} members (x{scale:.2f}); C++ restatement of the "
                                       "reference CPU solver"},
            "e2e": {"value": dt, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_reference(args, rank):
    if rank != 0:
        return
    db = build_workload(args.workload, max(args.steps, 8) + args.warmup + 8, scale=args.scale)
    n, dt, threads = time_oracle(db, max_steps=max(args.steps, 2), target_s=args.ref_seconds)
    value = db.nglob * n / dt
    line = {
        "metric": "GLL point-updates/s", "value": value, "unit": "point-updates/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": n, "warmup": 2, "ms_per_step": dt / n * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": {"workload": args.workload, "description": WORKLOAD_DESC[args.workload],
                                        "nspec": db.nspec, "nglob": db.nglob},
        "s_per_element_step": dt / n / db.nspec,
        "cpu_baseline": {"value": value, "unit": "point-updates/s", "cores": threads, "kind": "port",
                         "s_per_element_step": dt / n / db.nspec, "cpu_model": cpu_model(),
                         "sample": f"{n} Newmark steps of the full {db.nspec}-element mesh "
                                   "(C++ restatement of the reference CPU solver, FP32)"},
        "e2e": {"value": value, "unit": "point-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


FWI_WORKLOADS = {
    "c4_fwi_shots": ("misfit gradients of shots on the 1000x400-element (25 km x 10 km, 6,405,601 GLL points) "
                     "elastic model (vp 2500 m/s + 0.2 /s x depth, vs = vp/1.73, Gardner rho); Ricker 8 Hz "
                     "force 500 m deep at seeded surface positions (seed 5), 200 receivers, dt 4e-4, L2 misfit "
                     "against zero data (adjoint source = the synthetics: within 4000 steps no reflection "
                     "from the true model's anomalies, 3-7 km deep, reaches the receivers, so true-model data "
                     "would leave only rounding in the residual), checkpoint every 100 steps; batched = the "
                     "shots packed into meshes of --batch shots, plain = one shot per run"),
    "c5_fwi_models": ("misfit gradients of independent random-layered elastic models with uneven meshes "
                      "(sizes drawn with seed 6 between 100x50 and 1200x500 elements, 3-6 layers, vp 2000-4500, "
                      "one Ricker 8 Hz force, 20 surface receivers, dt 4e-4, Stacey on three sides); "
                      "L2 misfit against zero data (adjoint source = the synthetics), checkpoint every 100 steps; "
                      "batched = all models packed into one mesh and one launch per step, plain = one "
                      "model per run"),
}


def c4_shots(n_shots: int, nstep: int):
    """Shots of the C4 gradient workload on the starting model."""
    from specfem2d_b200 import batch, configs

    os.makedirs(CACHE, exist_ok=True)
    path = os.path.join(CACHE, f"c4_shots_{n_shots}_{nstep}.pkl")
    if os.path.exists(path):
        with open(path, "rb") as f:
            return pickle.load(f)
    xs = np.sort(np.random.default_rng(5).uniform(1000.0, 24000.0, n_shots))
    start = configs.c4_gradient(nstep=nstep)
    out = batch.shots_on_model(start, [(float(x), 9500.0) for x in xs])
    for d in out:
        d.mesh = None  # not needed past the source location
    with open(path, "wb") as f:
        pickle.dump(out, f)
    return out


def fwi_members(n_models: int, nstep: int, which: str = "first"):
    """The first n_models of the 48 seeded model sizes, or the n_models smallest."""
    from specfem2d_b200 import configs

    os.makedirs(CACHE, exist_ok=True)
    path = os.path.join(CACHE, f"c5_models_{which}_{n_models}_{nstep}.pkl")
    if os.path.exists(path):
        with open(path, "rb") as f:
            return pickle.load(f)
    sizes = list(enumerate(configs.c5_model_sizes()))
    if which == "smallest":
        sizes = sorted(sizes, key=lambda kv: kv[1][0] * kv[1][1])
    sizes = sizes[:n_models]
    models = [configs.random_layered_model(seed=100 + k, nx=nx, nz=nz, nstep=nstep) for k, (nx, nz) in sizes]
    with open(path, "wb") as f:
        pickle.dump(models, f)
    return models


def measure_coupled_gradient(db, checkpoint_every: int = 100):
    """Kernel run of a fluid-solid model through sf2d_coupled_fwi_* (forward
    with checkpoints, then the adjoint sweep with the forward segments
    recomputed; solid and fluid kernels): one untimed run, then one timed by
    the host clock around the C-ABI calls (traces in, kernels out included).
    The adjoint source is the synthetics themselves (zero observed data): the
    time does not depend on the data."""
    from specfem2d_b200.coupled import CoupledKernels

    k = CoupledKernels(db, checkpoint_every)
    try:
        k.backward(k.forward())
        t0 = time.perf_counter()
        seis = k.forward()
        t1 = time.perf_counter()
        kern = k.backward(seis)
        t2 = time.perf_counter()
    finally:
        k.close()
    ok = all(np.isfinite(v).all() for v in kern.values())
    return {"value": t2 - t0, "unit": "s per gradient", "forward_s": t1 - t0, "backward_s": t2 - t1,
            "nstep": db.nstep, "nglob": db.nglob, "checkpoint_every": checkpoint_every,
            "point_updates_per_s": 3.0 * db.nstep * db.nglob / (t2 - t0), "finite": bool(ok),
            "description": ("kernel run (forward, recomputed forward, adjoint; rho/kappa/mu in the solid, "
                            "rho/kappa in the water) of the c2 coupled model with Stacey sides and bottom, "
                            "host clock around sf2d_coupled_fwi_forward and _backward")}


def measure_fwi(args, all_models, nstep, world, rank, sum_shots=False):
    """Seconds per misfit gradient per model: plain (one model per run) and
    batched (the models packed into meshes of --batch members, one launch per
    step for all of them), both through sf2d_fwi_* with the traces and
    kernels copied to the host; models are sharded over the ranks."""
    import torch

    from specfem2d_b200 import batch
    from specfem2d_b200.distributed import max_over_ranks, shard, sum_over_ranks
    from specfem2d_b200.fwi import FWIGradient

    mine = shard([m.nspec for m in all_models], rank, world)
    models = [all_models[k] for k in mine]
    observed = [np.zeros((len(m.rec_ispec), nstep, 2)) for m in models]
    every = 100

    def one(db, obs):
        g = FWIGradient(db, every, tile_elems=args.tile_elems, threads_per_block=args.threads)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        seis = g.forward()
        kern = g.backward(seis - obs)
        t1 = time.perf_counter()
        g.close()
        return t1 - t0, kern

    plain_s = batched_s = num = den = 0.0
    local_nglob = 0
    if models:
        # warm-up on the smallest member (module load, graph instantiation)
        w = min(range(len(models)), key=lambda k: models[k].nspec)
        one(models[w], observed[w])
        plain_k = []
        for m, obs in zip(models, observed):
            t, k = one(m, obs)
            plain_s += t
            plain_k.append(k)
        bsize = args.batch if args.batch > 0 else len(models)
        bk = [[], [], []]
        for b0 in range(0, len(models), bsize):
            grp = models[b0:b0 + bsize]
            packed, idx = batch.pack(grp)
            local_nglob += packed.nglob
            t, kk = one(packed, np.concatenate(observed[b0:b0 + bsize], axis=0))
            batched_s += t
            for c in range(3):
                bk[c].extend(batch.split_elements(kk[c], idx))
        # gradient agreement: packed kernels against the per-model ones
        for c in range(3):
            for m, part in enumerate(bk[c]):
                ref = plain_k[m][c].astype(np.float64)
                num += float(np.sum((part.astype(np.float64) - ref) ** 2))
                den += float(np.sum(ref ** 2))
    summed = None
    if sum_shots:
        # shots of one model: the gradient of the summed misfit is the sum of the
        # shots' kernels, added on each rank and then over the ranks (NCCL)
        local = np.zeros((3,) + tuple(all_models[0].rhostore.shape), dtype=np.float64)
        for c in range(3):
            for part in (bk[c] if models else []):
                local[c] += part
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        total = sum_over_ranks(local, device="cuda")
        t_ar = max_over_ranks(time.perf_counter() - t0, device="cuda")
        summed = {"all_reduce_s": t_ar, "bytes": int(local.nbytes),
                  "max_abs": [float(np.abs(total[c]).max()) for c in range(3)]}
    plain_s = max_over_ranks(plain_s, device="cuda")
    batched_s = max_over_ranks(batched_s, device="cuda")
    num, den = (float(x) for x in sum_over_ranks(np.array([num, den]), device="cuda"))
    n = len(all_models)
    packed_nglob = int(sum_over_ranks(np.array([float(local_nglob)]), device="cuda")[0])
    return {"metric": "s per FWI gradient per shot", "unit": "s", "models": n, "steps": nstep,
            "sizes": [[int(m.nspec), int(m.nglob)] for m in all_models], "checkpoint_every": every,
            "plain_s_per_shot": plain_s / n, "batched_s_per_shot": batched_s / n,
            "speedup_batched_vs_plain": plain_s / batched_s,
            "gradient_rel_l2_batched_vs_plain": (num / den) ** 0.5 if den > 0 else 0.0,
            "point_updates_per_s_batched": 3.0 * packed_nglob * nstep / batched_s,
            "nglob_total": packed_nglob, "summed_gradient": summed}


def run_fwi(args, rank, world):
    """The FWI workloads as their own bench line (s per gradient per shot, batched)."""
    import torch

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    from specfem2d_b200.runtime import initialize_device

    initialize_device(int(os.environ.get("LOCAL_RANK", "0")))  # the library's own runtime, same device
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    if args.workload == "c4_fwi_shots":
        all_models = c4_shots(args.models, args.fwi_steps)
    else:
        all_models = fwi_members(args.models, args.fwi_steps, args.fwi_set)
    r = measure_fwi(args, all_models, args.fwi_steps, world, rank, sum_shots=args.workload == "c4_fwi_shots")
    line = {
        "metric": "s per FWI gradient per shot", "value": r["batched_s_per_shot"], "unit": "s", "n_gpus": world,
        "steps": args.fwi_steps, "warmup": 1, "higher_is_better": False, "scaling": "strong", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "description": FWI_WORKLOADS[args.workload], "models": r["models"],
                   "model_set": args.fwi_set, "sizes": r["sizes"],
                   "nspec_total": sum(m.nspec for m in all_models), "nglob_total": r["nglob_total"],
                   "checkpoint_every": r["checkpoint_every"],
                   "parallelism": f"models sharded over {world} GPU(s)",
                   "tile_elems": args.tile_elems, "threads_per_cta": args.threads},
        **{k: r[k] for k in ("plain_s_per_shot", "batched_s_per_shot", "speedup_batched_vs_plain",
                             "gradient_rel_l2_batched_vs_plain", "point_updates_per_s_batched",
                             "summed_gradient")},
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def measure_forward(db, args, workload, K, W, world, dist, nstep_full=0):
    """One forward workload: K graph-queued steps timed with CUDA events on the
    solver stream (max over ranks), per-kernel times for the roofline, and the
    end-to-end leg through the public API with pinned host buffers (K steps,
    and, with nstep_full, the configuration's whole run).  Returns the JSON
    fields of the workload."""
    import torch

    from specfem2d_b200.configs import (algorithmic_bytes_coupled, algorithmic_bytes_elastic,
                                        algorithmic_bytes_viscoelastic)
    from specfem2d_b200.coupled import CoupledSolver
    from specfem2d_b200.distributed import job_throughput, max_over_ranks
    from specfem2d_b200.runtime import ElasticSolver

    coupled = db.acoustic is not None
    tune = None
    if args.autotune:
        from specfem2d_b200.autotune import autotune_coupled, autotune_elastic

        if coupled:
            (args.fluid_tile_elems, args.pml_tile_elems, args.pml_threads), tune = autotune_coupled(
                db, args.tile_elems, args.threads)
        else:
            (args.tile_elems, args.threads), tune = autotune_elastic(db, tiles=(32, 48, 64), threads=(256, 512),
                                                                     steps=10, warmup=3)

    def make_solver():
        if coupled:
            return CoupledSolver(db, tile_elems=args.tile_elems, threads_per_block=args.threads,
                                 fluid_tile_elems=args.fluid_tile_elems, fluid_threads_per_block=args.fluid_threads,
                                 pml_tile_elems=args.pml_tile_elems, pml_threads_per_block=args.pml_threads)
        return ElasticSolver(db, tile_elems=args.tile_elems, threads_per_block=args.threads,
                             pml_tile_elems=args.pml_tile_elems, pml_threads_per_block=args.pml_threads)

    solver = make_solver()
    el_db = solver.sub_db if coupled else db   # the solid part the element-kernel roofline refers to
    stream = torch.cuda.ExternalStream(solver.stream_handle())

    # graph built and uploaded outside the timed region, warm-up, then the timed
    # region: K steps queued as CUDA graphs on the solver stream.  Fields and
    # element data exceed the 126 MB L2, so no flush is needed between steps.
    solver.prepare()
    solver.enqueue(W)
    solver.synchronize(600)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    time.sleep(0.3)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    solver.enqueue(K)
    ev1.record(stream)
    solver.synchronize(600)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = max_over_ranks(ev0.elapsed_time(ev1), device="cuda")  # the job lasts as long as its slowest rank
    if dist:
        dist.barrier()
    launches = solver.launch_count(K)

    # kernel-level timing for the roofline (events around each launch, same stream)
    nk = min(200, max(20, K // 10))
    k_ms = solver.time_kernels(nk)
    tile_ms = k_ms[2] if coupled else k_ms[0]
    shared_ms = k_ms[3] if coupled else k_ms[1]
    st = solver.solid_layout_info() if coupled else solver.layout_info()
    nsh = st["nshared"]
    n_int = el_db.nglob - nsh
    # algorithmic bytes of the (solid) element kernel per launch: element data + interior points
    # (u, v, a read+write, rmass) + shared points touched by tiles (u, v, a read, partial write)
    n_slots = st["n_slots"]
    pm = getattr(db, "pml", None)
    npml_el = int((el_db.pml["region"] > 0).sum()) if getattr(el_db, "pml", None) is not None else 0
    npml_ac = int((pm["region"] > 0).sum()) - npml_el if pm is not None else 0
    if db.atten is None:
        # + per CPML element point: damping profiles (48 B), rho J (4 B), memory variables read + write (96 B)
        tile_bytes = 700 * el_db.nspec + 56 * n_int + 32 * n_slots + 25 * 148 * npml_el
        step_bytes = algorithmic_bytes_elastic(db.nspec, db.nglob)
    elif db.time_scheme == 1:
        tile_bytes = 700 * db.nspec + 3600 * db.nspec + 56 * n_int + 32 * n_slots
        step_bytes = algorithmic_bytes_viscoelastic(db.nspec, db.nglob, 1)
    else:
        # per stage: element data, memory variables and their LDDRK copies, coefficients,
        # interior points (u, v, u_L, v_L read+write, a written, rmass read), shared reads + partial
        tile_bytes = db.nspec * (700 + 25 * 192) + 88 * n_int + 24 * n_slots
        step_bytes = algorithmic_bytes_viscoelastic(db.nspec, db.nglob, 2)
    if coupled:
        step_bytes = algorithmic_bytes_coupled(el_db.nspec, el_db.nglob, solver.nspec_fluid, solver.nglob_fluid,
                                               npml_el, npml_ac)
    traffic_key = (workload, args.tile_elems, args.threads, args.fluid_tile_elems, args.pml_tile_elems,
                   args.pml_threads)
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    achieved = tile_bytes / (tile_ms * 1e-3) / 1e9
    solver.close()

    def pinned(shape, dtype):
        return torch.zeros(shape, dtype=dtype).pin_memory().numpy()

    def e2e_run(nsteps):
        """Seconds (max over ranks) and bytes of one run through the public API:
        upload the initial fields, advance nsteps, read back the traces and the
        final fields, all through pinned host buffers.  The solver and its step
        graph are set up before the timed region, as the reference's
        prepare_*_device calls are."""
        sol = make_solver()
        sol.prepare()
        zeros = pinned((db.nglob, 2), torch.float32)
        seis_buf = pinned((sol.nrec, nsteps, 2), torch.float64)
        if coupled:
            z1 = pinned((db.nglob,), torch.float32)
            outs = {k: pinned((db.nglob, 2), torch.float32) for k in ("displ", "veloc", "accel")}
            outs.update({k: pinned((db.nglob,), torch.float32) for k in ("pot", "pot_dot", "pot_dot_dot")})
        else:
            outs = [pinned((db.nglob, 2), torch.float32) for _ in range(3)]
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        if coupled:
            sol.set_fields(displ=zeros, veloc=zeros, accel=zeros, pot=z1, pot_dot=z1, pot_dot_dot=z1)
            seis = sol.run(nsteps, seismograms=True, out=seis_buf)
            sol.get_fields(out=outs)
            h2d = 3 * db.nglob * 8 + 3 * db.nglob * 4
        else:
            sol.set_fields(zeros, zeros, zeros)
            seis = sol.run(nsteps, seismograms=True, out=seis_buf)
            sol.get_fields(out=outs)
            h2d = 3 * db.nglob * 8
        t1 = time.perf_counter()
        d2h = seis.nbytes + h2d  # the traces and the same fields read back
        sol.close()
        return max_over_ranks(t1 - t0, device="cuda"), h2d, d2h

    e2e = None
    if not args.no_e2e:
        e2e_s, h2d, d2h = e2e_run(K)
        e2e = {"value": db.nglob * K * world / e2e_s, "unit": "point-updates/s",
               "h2d_bytes_per_step": h2d / K, "d2h_bytes_per_step": d2h / K}
    e2e_full = None
    if nstep_full and not args.no_e2e:
        e2e_s, h2d, d2h = e2e_run(nstep_full)
        e2e_full = {"value": db.nglob * nstep_full * world / e2e_s, "unit": "point-updates/s", "steps": nstep_full,
                    "seconds": e2e_s, "h2d_bytes_per_step": h2d / nstep_full, "d2h_bytes_per_step": d2h / nstep_full}

    value = job_throughput(db.nglob * K, ms * 1e-3, world, device="cuda")
    return {
        "value": value, "ms_per_step": ms / K,
        "config": {"workload": workload, "description": WORKLOAD_DESC[workload], "scale": args.scale,
                   "nspec": db.nspec, "nglob": db.nglob, "tile_elems": args.tile_elems,
                   "fluid_tile_elems": (args.fluid_tile_elems or args.tile_elems) if coupled else None,
                   "fluid_threads_per_cta": (args.fluid_threads or args.threads) if coupled else None,
                   "cpml_tile_elems": args.pml_tile_elems or args.tile_elems,
                   "cpml_threads_per_cta": args.pml_threads or args.threads,
                   "threads_per_cta": args.threads, "autotuned": bool(tune),
                   "autotune_candidates": tune,
                   "ntiles": st["ntiles"], "shared_points": nsh,
                   "nspec_fluid": solver.nspec_fluid if coupled else 0,
                   "cpml_elements": {"solid": npml_el, "fluid": npml_ac},
                   "l2": "inputs larger than L2 (fields + element data > 126 MB), no flush needed",
                   "e2e_setup": "solver created and step graph built before the timed region; "
                                "fields and traces through pinned host buffers",
                   "parallelism": f"replicas x{world}"},
        "hbm_gbs_step": step_bytes / (ms / K * 1e-3) / 1e9,
        # the reference's logs quote time per spectral element and step; local
        # point-updates count every element GLL point (25 nspec per step)
        "local_point_updates_per_s": 25 * db.nspec * K * world / (ms * 1e-3),
        "s_per_element_step": ms * 1e-3 / K / db.nspec,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": TILE_TRAFFIC.get(traffic_key),
                     "traffic_source": TRAFFIC_SOURCE.get(traffic_key),
                     "kernel": "k_elastic_tile", "kernel_ms": tile_ms, "shared_kernel_ms": shared_ms,
                     "fluid_kernels_ms": k_ms[:2] if coupled else None, "step_kernels_ms": k_ms[-1],
                     "algorithmic_bytes_per_launch": tile_bytes,
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if peaks else "fallback"},
        "e2e": e2e, "e2e_full_run": e2e_full,
        "gpu_launches": launches,
        "clocks": clk,
    }


def cpu_model() -> str:
    """The host CPU's model name (/proc/cpuinfo), recorded beside the CPU baseline."""
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c3_viscoelastic", choices=sorted(WORKLOAD_DESC) + sorted(FWI_WORKLOADS))
    ap.add_argument("--models", type=int, default=12, help="models of the FWI workload")
    ap.add_argument("--fwi-steps", type=int, default=1000, help="time steps of each FWI model")
    ap.add_argument("--fwi-set", default="first", choices=["first", "smallest"],
                    help="the first --models of the 48 seeded sizes, or the smallest")
    ap.add_argument("--batch", type=int, default=0, help="members per packed mesh in the FWI workloads (0 = all)")
    ap.add_argument("--tile-elems", type=int, default=32)
    ap.add_argument("--threads", type=int, default=256)
    ap.add_argument("--fluid-tile-elems", type=int, default=64, help="fluid tiles (coupled runs); 0 = --tile-elems")
    ap.add_argument("--fluid-threads", type=int, default=0, help="fluid CTA threads; 0 = --threads")
    ap.add_argument("--pml-tile-elems", type=int, default=16, help="solid CPML tiles; 0 = --tile-elems")
    ap.add_argument("--pml-threads", type=int, default=128, help="solid CPML CTA threads; 0 = --threads")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="keep the given tile options instead of tuning them first")
    ap.add_argument("--ref-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end legs (profiling runs)")
    ap.add_argument("--no-extras", action="store_true",
                    help="headline workload only (no C2 coupled and batched-gradient keys)")
    ap.add_argument("--scale", type=int, default=1,
                    help="divide the element counts of the c2/c3 workloads (small profiling cases only)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.workload in FWI_WORKLOADS:
        if args.impl == "reference":
            run_reference_fwi(args, rank)
        else:
            run_fwi(args, rank, world)
        return
    if args.impl == "reference":
        run_reference(args, rank)
        return

    import torch

    torch.cuda.set_device(local_rank)
    from specfem2d_b200.runtime import initialize_device

    initialize_device(local_rank)  # the library's own CUDA runtime on the same device
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist_mod

        dist_mod.init_process_group("nccl", timeout=datetime.timedelta(seconds=900))
        dist = dist_mod

    K, W = args.steps, args.warmup
    full = WORKLOAD_NSTEP.get(args.workload, 0) if args.scale == 1 else 0
    db = build_workload(args.workload, max(K + W + 8, full), rank=rank, dist=dist, scale=args.scale)
    base_args = copy.copy(args)
    res = measure_forward(db, args, args.workload, K, W, world, dist, nstep_full=full if world == 1 else 0)
    line = {"metric": "GLL point-updates/s", "value": res["value"], "unit": "point-updates/s",
            "n_gpus": world, "steps": K, "warmup": W, "ms_per_step": res["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", **{k: res[k] for k in ("config", "hbm_gbs_step", "local_point_updates_per_s",
                                                          "s_per_element_step", "roofline", "e2e",
                                                          "e2e_full_run", "gpu_launches", "clocks")}}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        n, dt, threads = time_oracle(db, max_steps=K, target_s=args.ref_seconds)
        line["cpu_baseline"] = {"value": db.nglob * n / dt, "unit": "point-updates/s", "cores": threads,
                                "kind": "port", "s_per_element_step": dt / n / db.nspec,
                                "cpu_model": cpu_model(),
                                "sample": f"{n} time steps of the full mesh, C++ restatement of the "
                                          "reference CPU solver (FP32), all host threads"}
    del db
    if world == 1 and not args.no_extras and args.scale == 1:
        # the other configurations of the metric, as extra keys of the same line,
        # each tuned from the command line's tile options
        c2 = build_workload("c2_coupled", K + W + 8)
        r2 = measure_forward(c2, copy.copy(base_args), "c2_coupled", K, W, world, dist)
        line["c2_coupled"] = {"value": r2["value"], "unit": "point-updates/s", "ms_per_step": r2["ms_per_step"],
                              "nglob": c2.nglob, "roofline_frac": r2["roofline"]["frac"],
                              "tiles": {k: r2["config"][k] for k in ("tile_elems", "threads_per_cta",
                                                                      "fluid_tile_elems", "cpml_tile_elems",
                                                                      "cpml_threads_per_cta")},
                              "autotune_candidates": r2["config"]["autotune_candidates"],
                              "tile_kernel_ms": r2["roofline"]["kernel_ms"], "e2e": r2["e2e"],
                              "clocks": r2["clocks"]}
        del c2
        members = fwi_members(24, 400, "smallest")
        fargs = copy.copy(base_args)
        btune = None
        if fargs.autotune:
            from specfem2d_b200.autotune import autotune_batch

            obs = [np.zeros((len(m.rec_ispec), 400, 2)) for m in members]
            fargs.batch, btune = autotune_batch(members, obs, sizes=(1, 4, 8, 24), sample=24)
        fwi = measure_fwi(fargs, members, 400, world, rank)
        fwi["members_per_batch"] = fargs.batch or len(members)
        fwi["autotune_candidates"] = btune
        fwi["description"] = ("the c5_fwi_models workload on its 24 smallest models (5,450-149,151 elements), "
                              "400 steps: " + FWI_WORKLOADS["c5_fwi_models"])
        line["fwi_gradient"] = fwi
        c2s = build_workload("c2_coupled_stacey", 400)
        line["fluid_solid_gradient"] = measure_coupled_gradient(c2s, 100)
        del c2s
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
