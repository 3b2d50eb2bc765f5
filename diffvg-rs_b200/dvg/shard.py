"""Multi-process plumbing for running the hot path on several GPUs.

The path shards by scene: every rank renders and differentiates its own scenes,
with no exchange in the data path (weak scaling).  What the ranks share is
bookkeeping: which scenes a rank owns, per-rank seeds, and the step time, which
is the maximum over ranks of each rank's CUDA-event time.  Everything here runs
on any torch.distributed backend (NCCL on GPUs, gloo on CPU for tests).
"""
from __future__ import annotations

from typing import List, Sequence, Tuple


def shard_range(n: int, rank: int, world: int) -> Tuple[int, int]:
    """Contiguous, balanced [begin, end) of n units owned by `rank` (the first n % world
    ranks take one extra unit)."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("rank out of range")
    base, extra = divmod(n, world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def rank_seed(seed: int, rank: int) -> int:
    """Seed of a rank's scenes: distinct per rank, reproducible from (seed, rank)."""
    return (seed * 1_000_003 + rank) & 0x7FFFFFFF


def max_over_ranks(values: Sequence[float], device="cpu") -> List[float]:
    """Element-wise maximum of `values` over all ranks (identity without a process group)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [float(v) for v in values]
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu()]


def weak_scaling_rate(units_per_rank: float, world: int, max_ms: float) -> float:
    """Whole-job throughput in units per second when every rank did `units_per_rank`
    units and the slowest rank took `max_ms`."""
    return units_per_rank * world / (max_ms / 1e3)
