"""Replica plumbing for several GPUs of one node: every rank builds its own
share of independent reconstructors (no collective on the data path); the only
collectives are the barrier around the timed region and one reduction of the
timing (the max over ranks) and of the unit counts."""
from __future__ import annotations

from typing import List, Sequence


def shard(units: Sequence, rank: int, world: int) -> List:
    """Round-robin share of `units` for `rank` (every unit exactly once)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("shard: bad rank/world")
    return list(units[rank::world])


def max_over_ranks(x: float, dist=None, device: str = "cpu") -> float:
    """The maximum of x over all ranks (x itself without a process group)."""
    if dist is None or not dist.is_initialized():
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, dist=None, device: str = "cpu") -> float:
    if dist is None or not dist.is_initialized():
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def whole_job_rate(units_done: float, seconds_local: float, dist=None, device: str = "cpu") -> float:
    """Units processed by all ranks divided by the slowest rank's time."""
    total = sum_over_ranks(units_done, dist, device)
    slowest = max_over_ranks(seconds_local, dist, device)
    return total / slowest
