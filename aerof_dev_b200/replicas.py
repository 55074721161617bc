"""Replica runs over several GPUs (one process per GPU, torch.distributed).

The path does not shard in this build: every rank evaluates the same-size
problem on its own GPU with no data-path collective.  The only exchange is
the timing reduction: the job's time is the slowest rank's device time, and
its throughput counts the work of every rank.
"""
from __future__ import annotations


def max_over_ranks(value: float, device: str = "cpu") -> float:
    """The maximum of ``value`` over all ranks of the default process group
    (the value itself when no group is initialised).  ``device`` is where the
    reduction tensor lives: "cuda" for NCCL, "cpu" for gloo."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(units_per_rank: float, world: int, ms: float) -> float:
    """Whole-job rate in units per second: every rank's units over the
    slowest rank's time (weak scaling)."""
    return units_per_rank * world / (ms * 1e-3)
