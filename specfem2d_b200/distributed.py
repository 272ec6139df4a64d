"""Host-side plumbing for runs on several GPUs of one node (one process per GPU).

The forward path of one mesh does not shard in this design: several GPUs run
independent replicas (benchmark) or independent shots and models (misfit
gradients), so the only collectives are a maximum of device times over ranks
and one sum of sensitivity kernels at the end of a gradient batch.  All of
them go through torch.distributed (NCCL on GPUs, gloo on CPU); without an
initialised process group every helper returns its input unchanged.
"""
from __future__ import annotations

import numpy as np


def _dist():
    import torch.distributed as dist

    return dist if dist.is_available() and dist.is_initialized() else None


def rank_world() -> tuple[int, int]:
    d = _dist()
    return (d.get_rank(), d.get_world_size()) if d else (0, 1)


def shard(costs, rank: int, world: int) -> list[int]:
    """Indices of the items this rank runs: a greedy longest-first split of
    `costs` (one per item, e.g. element counts) into `world` parts of nearly
    equal total cost.  Every rank computes the same split; every item lands on
    exactly one rank."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank or world size")
    order = sorted(range(len(costs)), key=lambda k: (-float(costs[k]), k))
    load = [0.0] * world
    owner = [0] * len(costs)
    for k in order:
        r = min(range(world), key=lambda q: (load[q], q))
        owner[k] = r
        load[r] += float(costs[k])
    return [k for k in range(len(costs)) if owner[k] == rank]


def max_over_ranks(x: float, device: str = "cpu") -> float:
    """Maximum of a scalar over all ranks (device times: the job takes as long as its slowest rank)."""
    d = _dist()
    if d is None:
        return float(x)
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    d.all_reduce(t, op=d.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(a, device: str = "cpu"):
    """Element-wise sum of an array over all ranks (kernels of shots split over GPUs)."""
    d = _dist()
    arr = np.asarray(a)
    if d is None:
        return arr
    import torch

    t = torch.from_numpy(np.ascontiguousarray(arr, dtype=np.float64)).to(device)
    d.all_reduce(t, op=d.ReduceOp.SUM)
    return t.cpu().numpy().astype(arr.dtype, copy=False)


def job_throughput(units_per_rank: float, seconds_per_rank: float, world: int, device: str = "cpu") -> float:
    """Whole-job rate of weak-scaled replicas: all ranks' units over the slowest rank's time."""
    t = max_over_ranks(seconds_per_rank, device)
    return units_per_rank * world / t
