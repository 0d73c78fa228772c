"""Replicas: one independent fluid world per GPU, one process per GPU.

The fluid step has no exchange step that shards (a slab split would trade halos after every
globally synchronised pass), so `bench.py --gpus N` runs N independent worlds.  The only
collectives are the measurement's own: a barrier around the timed region and this reduction of
each rank's work and device time.
"""
from __future__ import annotations


def reduce_timing(substeps: int, ms: float, world_size: int, device=None) -> tuple[int, float]:
    """(substeps summed over the ranks, the slowest rank's device milliseconds).

    The job's throughput is the first over the second: every replica's work, finished when the
    slowest replica finishes.  With one rank nothing is exchanged.
    """
    if world_size == 1:
        return int(substeps), float(ms)
    import torch
    import torch.distributed as dist

    work = torch.tensor([float(substeps)], dtype=torch.float64, device=device)
    slowest = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(work, op=dist.ReduceOp.SUM)
    dist.all_reduce(slowest, op=dist.ReduceOp.MAX)
    return int(round(work.item())), float(slowest.item())
