"""Multi-GPU runs of the network-to-conductance path: independent replicas.

One network's systems are too small to split across GPUs (its solve is
latency-bound on one), so N GPUs solve N independent seeded networks, one
process per GPU; a Monte-Carlo sweep splits its realisations over the ranks
(`shard`).  The only collectives are the timing barrier and the reductions of
the measured times and counts (NCCL on GPUs, gloo on CPU); the data path has
none.
"""
from __future__ import annotations

import datetime
import os


def env():
    """(rank, world size, local rank) from the torchrun environment."""
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def seed(rank: int, base: int = 2_000_000) -> int:
    """Seed of the network replica `rank` solves."""
    return base + rank


def init(world: int, gpu: bool, timeout_s: int = 600):
    """Create the process group when world > 1 (nccl with GPUs, gloo without)."""
    if world <= 1:
        return
    import torch.distributed as dist

    if not dist.is_initialized():
        dist.init_process_group("nccl" if gpu else "gloo", timeout=datetime.timedelta(seconds=timeout_s))


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(values, world: int, device=None):
    """Element-wise maximum of a list of floats over all ranks."""
    if world <= 1:
        return [float(v) for v in values]
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu()]


def sum_over_ranks(values, world: int, device=None):
    """Element-wise sum of a list of floats over all ranks."""
    if world <= 1:
        return [float(v) for v in values]
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return [float(v) for v in t.cpu()]


def shard(items, sizes, rank: int, world: int):
    """The items rank `rank` takes when independent work items (Monte-Carlo
    realisations) are split over `world` ranks: largest first, dealt round-robin,
    so the ranks' totals stay close; every item goes to exactly one rank."""
    order = sorted(range(len(items)), key=lambda k: (-sizes[k], k))
    return [items[k] for k in order[rank::world]]


def sweep_totals(seconds: float, count: float, failed: bool, world: int, device=None):
    """(slowest rank's seconds, total count, any rank failed) of a sharded sweep.
    Every rank calls it once, also when its own shard failed, so all ranks take
    the same collective steps."""
    t = max_over_ranks([seconds, 1.0 if failed else 0.0], world, device)
    n = sum_over_ranks([count], world, device)
    return t[0], n[0], t[1] > 0


def finish(world: int):
    if world > 1:
        import torch.distributed as dist

        if dist.is_initialized():
            dist.destroy_process_group()
