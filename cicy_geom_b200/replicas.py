"""Multi-GPU runs of the network-to-conductance path: independent replicas.

One network's systems are too small to split across GPUs (its solve is
latency-bound on one), so N GPUs solve N independent seeded networks, one
process per GPU.  The only collectives are the timing barrier and the
max-over-ranks of the measured times (NCCL on GPUs, gloo on CPU); the data
path has none.
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


def finish(world: int):
    if world > 1:
        import torch.distributed as dist

        if dist.is_initialized():
            dist.destroy_process_group()
