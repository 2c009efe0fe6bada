"""Replica plumbing of the multi-GPU bench: one independent case per rank.

The substep has no exchange between ranks (each rank advances its own case,
seeded by its rank), so the only collectives are the timing reductions:
the timed region's length is the maximum over ranks, and the whole-job
throughput counts the points all ranks advanced in that time.
"""
from __future__ import annotations


def case_seed(rank: int) -> int:
    """Seed of the initial condition of rank's case."""
    return int(rank)


def max_over_ranks(x: float, dist=None, device="cpu") -> float:
    """The maximum of x over all ranks (x itself without a process group)."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(mpts_per_case: float, steps: int, world: int, seconds: float) -> float:
    """Whole-job Mpts*steps/s: every rank advanced its case by `steps`."""
    return mpts_per_case * steps * world / seconds
