"""The multi-process plumbing of bench.py and of sharded gradient batches,
run as two gloo ranks on the CPU: shard assignment, max-over-ranks device
time, whole-job throughput of weak-scaled replicas, sum of kernels."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    from specfem2d_b200 import distributed as D

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        assert D.rank_world() == (rank, world)
        # replicas: rank r took (1 + r) seconds for 1000 units
        t = D.max_over_ranks(1.0 + rank)
        rate = D.job_throughput(1000.0, 1.0 + rank, world)
        # kernels of the shots each rank ran, summed over ranks
        costs = [5, 1, 7, 3, 3, 9, 2]
        mine = D.shard(costs, rank, world)
        k = np.zeros(len(costs))
        for i in mine:
            k[i] = costs[i] * 10.0 + rank
        total = D.sum_over_ranks(k)
        out[rank] = (t, rate, mine, total.tolist())
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    costs = [5, 1, 7, 3, 3, 9, 2]
    for r in range(world):
        t, rate, mine, total = res[r]
        assert t == 2.0                          # the slowest rank's time
        assert rate == pytest.approx(1000.0 * world / 2.0)
    owned = sorted(res[0][2] + res[1][2])
    assert owned == list(range(len(costs)))     # every shot on exactly one rank
    loads = [sum(costs[i] for i in res[r][2]) for r in range(world)]
    assert abs(loads[0] - loads[1]) <= max(costs)
    expect = [costs[i] * 10.0 + (0 if i in res[0][2] else 1) for i in range(len(costs))]
    assert res[0][3] == expect and res[1][3] == expect


def test_single_process_helpers_pass_through():
    from specfem2d_b200 import distributed as D

    assert D.rank_world() == (0, 1)
    assert D.max_over_ranks(3.5) == 3.5
    a = np.arange(4.0)
    assert np.array_equal(D.sum_over_ranks(a), a)
    assert D.shard([1, 2, 3], 0, 1) == [0, 1, 2]
    with pytest.raises(ValueError):
        D.shard([1], 2, 2)
