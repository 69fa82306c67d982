"""Replica sharding of the analysis across GPUs (one process per GPU, no data-path collective).

Pictures of one clip depend on each other (the wavefront inside a picture, the reconstruction
chain across a GOP), so the unit of distribution is the clip: rank r analyses its own clip,
seeded by r, and the only collective is the reduction of the timing. The whole-job rate is the
work of all ranks over the slowest rank's time.
"""
from __future__ import annotations


def clip_seed(rank: int) -> int:
    """Seed of the synthetic clip rank `rank` analyses (distinct per rank)."""
    return 2 + rank


def slowest(seconds: float, world: int, device="cpu") -> float:
    """The largest `seconds` over all ranks (all ranks must call it, in the same order)."""
    if world <= 1:
        return float(seconds)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(seconds)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: float, seconds: float, world: int, device="cpu") -> float:
    """Units per second of the whole job: world * units over the slowest rank's time."""
    worst = slowest(seconds, world, device)
    return world * units_per_rank / worst if worst > 0 else 0.0
