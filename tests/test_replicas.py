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


def test_single_process_needs_no_group():
    from cicy_geom_b200 import replicas as R

    R.init(1, gpu=False)
    assert R.max_over_ranks([3.0], 1) == [3.0]
    assert R.seed(3) == 2_000_003
