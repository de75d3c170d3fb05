"""Replica plumbing of multi-GPU runs (cicy_geom_b200/replicas.py), on CPU with
the gloo backend and two ranks: distinct seeds, the timing barrier and the
max-over-ranks reduction that `bench.py --gpus N` uses."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank), "MASTER_ADDR": "127.0.0.1",
                       "MASTER_PORT": str(port)})
    from cicy_geom_b200 import replicas as R

    r, w, l = R.env()
    R.init(w, gpu=False, timeout_s=60)
    R.barrier(w)
    t = R.max_over_ranks([1.0 + r, 10.0 - r], w)
    out[r] = (R.seed(r), t)
    R.finish(w)


def test_two_replicas_gloo():
    world, port = 2, _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    seeds = {out[r][0] for r in range(world)}
    assert len(seeds) == world  # every replica solves its own network
    for r in range(world):
        assert out[r][1] == [2.0, 10.0]  # max over ranks, element-wise
    # whole-job throughput from the slowest rank, as bench.py reports it
    steps, t_max = 5, out[0][1][0]
    assert world * steps / t_max == pytest.approx(5.0)


def _sweep_rank(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank), "MASTER_ADDR": "127.0.0.1",
                       "MASTER_PORT": str(port)})
    from cicy_geom_b200 import replicas as R

    R.init(world, gpu=False, timeout_s=60)
    sizes = [5, 40, 12, 33, 7, 21, 18]
    mine = R.shard(list(range(len(sizes))), sizes, rank, world)
    # rank 1 "fails" its shard; both ranks still take the same reductions
    t, n, failed = R.sweep_totals(1.5 + rank, float(len(mine)), failed=(rank == 1), world=world)
    out[rank] = (mine, t, n, failed)
    R.finish(world)


def test_monte_carlo_sweep_sharded_over_two_ranks_gloo():
    world, port = 2, _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_sweep_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    shards = [out[r][0] for r in range(world)]
    assert sorted(shards[0] + shards[1]) == list(range(7))  # every realisation on exactly one rank
    assert shards[0] == [1, 5, 2, 0] and shards[1] == [3, 6, 4]  # sizes 40, 33, 21, 18, 12, 7, 5 dealt round-robin
    for r in range(world):
        assert out[r][1:] == (2.5, 7.0, True)  # slowest rank, total count, the failure seen by every rank


def _bench_sweep_rank(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank), "MASTER_ADDR": "127.0.0.1",
                       "MASTER_PORT": str(port)})
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    from cicy_geom_b200 import replicas as R

    R.init(world, gpu=False, timeout_s=60)
    out[rank] = bench.sharded_monte_carlo(4, rank, rank, world)
    R.finish(world)


def test_bench_sharded_sweep_ranks_finish_together_when_shards_fail():
    # no GPU here: every rank's shard fails, and every rank still completes the same reductions
    import torch

    if torch.cuda.is_available():
        pytest.skip("checks the failure path, which needs a machine without a GPU")
    world, port = 2, _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_bench_sweep_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
        assert p.exitcode == 0
    for r in range(world):
        assert out[r]["failed_on_some_rank"] is True and out[r]["systems"] == 0 and out[r]["ranks"] == world


def test_single_process_needs_no_group():
    from cicy_geom_b200 import replicas as R

    R.init(1, gpu=False)
    assert R.max_over_ranks([3.0], 1) == [3.0]
    assert R.seed(3) == 2_000_003
