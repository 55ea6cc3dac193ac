"""Process-per-GPU plumbing for independent replicas (no collective on the
data path: each rank advances its own system; only timings are combined).

BD_BOX runs one system per process and has no GPU decomposition of a single
system that this library reproduces, so several GPUs run independent
replicas. torch.distributed is used for the rendezvous, one barrier around
the timed region and the max-over-ranks of the measured time.
"""
from __future__ import annotations

import datetime
import os


def init(backend: str = "nccl", timeout_s: int = 120):
    """(dist or None, rank, world, local_rank) from the torchrun environment."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world <= 1:
        return None, 0, 1, local
    import torch.distributed as dist
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist, rank, world, local


def replica_seed(base: int, rank: int) -> int:
    """Noise key of rank's replica: distinct per rank, fixed per run."""
    return base + 1000 * rank


def max_over_ranks(dist, value: float, device: str = "cpu") -> float:
    """The largest value over all ranks (the job's time is its slowest rank's)."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist):
    if dist is not None:
        dist.barrier()


def finish(dist):
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
