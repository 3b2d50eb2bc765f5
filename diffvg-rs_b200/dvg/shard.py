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


def cost_range(costs: Sequence[float], rank: int, world: int) -> Tuple[int, int]:
    """Contiguous [begin, end) of the units (in order) owned by `rank`, cut where the
    running cost crosses k/world of the total, so that every rank gets about the same
    cost rather than the same count.  The ranges of ranks 0..world-1 cover every unit
    exactly once, in order (some may be empty when a few units carry all the cost)."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("rank out of range")
    n = len(costs)
    prefix = [0.0]
    for c in costs:
        prefix.append(prefix[-1] + max(float(c), 0.0))
    total = prefix[-1]
    if total <= 0.0:
        return shard_range(n, rank, world)

    def cut(k):  # first unit index whose prefix reaches k/world of the total
        if k <= 0:
            return 0
        if k >= world:
            return n
        goal = total * k / world
        lo, hi = 0, n
        while lo < hi:
            mid = (lo + hi) // 2
            if prefix[mid + 1] - 0.5 * max(float(costs[mid]), 0.0) < goal:  # unit mid's midpoint before the goal
                lo = mid + 1
            else:
                hi = mid
        return lo
    return cut(rank), cut(rank + 1)


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


class SceneShardStep:
    """One scene split over `world` processes: forward + L2 loss + backward of a band
    of tiles and a range of boundary samples per process, with two sums across
    processes (the splat accumulators after the forward, the gradients after the
    backward).  Tiles are split by cost (balance=True, cost_range over the groups
    binned to each tile) or by count.  `all_reduce(tensor)` sums a device tensor over
    the processes in place (torch.distributed.all_reduce over NCCL on GPUs; run step() with the library's
    stream as torch's current stream so the collectives follow its kernels).  After
    step() every process holds the whole image, the loss and the whole scene's
    gradients in `grads`."""

    def __init__(self, scene, options, bopts, rank: int, world: int, all_reduce, device="cuda", balance=True):
        import torch

        from .renderer import DeviceGrads
        from .scene import BackwardOptions

        self.scene, self.options = scene, options
        self.bopts = bopts or BackwardOptions()
        self.all_reduce = all_reduce
        w, h = scene.scene.width, scene.scene.height
        self.npix = w * h
        # tiles split by cost (groups binned to the tile, plus one for its sampling and
        # splat), not by count: tile bands of one scene can differ widely in work
        self.tiles = cost_range([g + 1 for g in scene.tile_groups()], rank, world) if balance else \
            shard_range(scene.tile_count(), rank, world)
        nb = self.bopts.boundary_samples or self.npix * options.samples_x * options.samples_y
        self.samples = shard_range(nb, rank, world)
        # accumulators in one buffer (RGBA sums, then weights): one collective
        self.acc = torch.zeros(self.npix * 5, dtype=torch.float32, device=device)
        self.image = torch.zeros(self.npix * 4, dtype=torch.float32, device=device)
        self.d_render = torch.zeros(self.npix * 4, dtype=torch.float32, device=device)
        self.loss = torch.zeros(1, dtype=torch.float32, device=device)
        self.grads = DeviceGrads(scene.packed, device)

    def step(self, target) -> None:
        s, acc = self.scene, self.acc
        accum_ptr, wsum_ptr = acc.data_ptr(), acc.data_ptr() + self.npix * 16
        s.shard_forward(self.options, self.tiles, accum_ptr, wsum_ptr)
        self.all_reduce(acc)
        s.shard_resolve(accum_ptr, wsum_ptr, self.image.data_ptr())
        s.renderer.l2_device(self.image.data_ptr(), target.data_ptr(), self.npix * 4, self.d_render.data_ptr(),
                             self.loss.data_ptr())
        s.shard_backward(self.options, self.bopts, self.tiles, self.samples, self.d_render.data_ptr(), wsum_ptr,
                         self.grads)
        self.all_reduce(self.grads.buffer)
