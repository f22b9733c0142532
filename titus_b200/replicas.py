"""Multi-GPU aggregation for replica runs.

A single dose solve does not shard: a multi-GPU run is N independent solves,
one per rank (one process per GPU), with no data exchange. Whole-job
throughput is the units all ranks processed divided by the slowest rank's
device time (max over ranks).
"""
from __future__ import annotations


def max_over_ranks(seconds: float, device=None) -> float:
    """Max of a per-rank time over the default process group (identity when
    torch.distributed is not initialised). Every rank must call it."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return float(seconds)
    t = torch.tensor([float(seconds)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(units_per_rank: float, seconds: float, world: int, device=None):
    """(whole-job units/s, max-over-ranks seconds) for `world` replicas."""
    t = max_over_ranks(seconds, device)
    return world * units_per_rank / t, t
