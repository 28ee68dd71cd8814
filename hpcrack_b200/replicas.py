"""Multi-GPU execution as independent replicas (one specimen per rank, weak scaling).

A staggered fracture solve of one specimen runs on one GPU; N GPUs solve N specimens with no
data-path collective.  The only cross-rank traffic is the timing/aggregation below: the job's
time is the maximum over ranks of the device-timed region, its work the sum of the ranks' work.
The helpers work with any torch.distributed backend (NCCL on GPUs, gloo on CPU for tests).
"""
from __future__ import annotations

import os


def rank_info():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def replica_seed(base_seed: int, rank: int, distinct: bool) -> int:
    """Seed of the specimen a rank solves: identical replicas by default, distinct when asked."""
    return base_seed + (1000 * rank if distinct else 0)


def _device_for_backend():
    import torch
    import torch.distributed as dist
    if dist.is_initialized() and dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def aggregate(elapsed_ms: float, work: float, world: int):
    """(max elapsed over ranks, summed work) - every rank takes the same collective steps."""
    if world == 1:
        return elapsed_ms, work
    import torch
    import torch.distributed as dist
    dev = _device_for_backend()
    t = torch.tensor([elapsed_ms], dtype=torch.float64, device=dev)
    w = torch.tensor([work], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(w, op=dist.ReduceOp.SUM)
    return float(t.item()), float(w.item())


def throughput(elapsed_ms: float, work: float, world: int) -> float:
    """Whole-job throughput in work units per second (the max-over-ranks clock)."""
    t, w = aggregate(elapsed_ms, work, world)
    return w / (t / 1e3)


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
