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


def _grad_worker(rank, world, port, out):
    import datetime
    import sys

    import torch.distributed as dist

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in (root, os.path.join(root, "oracle"), os.path.join(root, "tests")):
        if p not in sys.path:
            sys.path.insert(0, p)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        out[rank] = _survey_gradient()
    finally:
        dist.destroy_process_group()


def _survey_gradient():
    """Summed gradient of three shots on the small inversion case, computed with
    the FP64 oracle in place of the GPU."""
    import oracle

    from fwi_case import Case
    from specfem2d_b200 import batch
    from specfem2d_b200.fwi import summed_shot_gradient

    c = Case(nstep=300)
    shots = batch.shots_on_model(c.start_db(), [(1000.0, 1800.0), (2000.0, 1500.0), (3000.0, 1900.0)], 30.0)
    truth = batch.shots_on_model(c.true_db(), [(1000.0, 1800.0), (2000.0, 1500.0), (3000.0, 1900.0)], 30.0)
    observed = [oracle.Oracle(t, 8).run(t.nstep) for t in truth]

    def grad(db, obs):
        return oracle.gradient(db, obs, checkpoint_every=100, precision=8)

    chi, rk, kk, mk = summed_shot_gradient(shots, observed, gradient_fn=grad)
    return chi, rk, kk, mk


def test_summed_shot_gradient_over_two_gloo_ranks():
    """The shots of one model split over two ranks, each rank's kernels summed,
    one all-reduce: the same gradient as one process running every shot (up to
    the order of the sums)."""
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_grad_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    single = _survey_gradient()
    for r in range(world):
        assert res[r][0] == pytest.approx(single[0], rel=1e-12)
        for a, b in zip(res[r][1:], single[1:]):
            assert np.allclose(a, b, rtol=1e-12, atol=1e-12 * np.abs(b).max())
    # every shot's kernels are in the sum: the three-shot sum is not one shot's
    assert np.abs(single[1]).max() > 0
