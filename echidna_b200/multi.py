"""Multi-GPU sharding of batched sweeps: one process per GPU.

Points are independent, so a batch is split into contiguous point ranges, one
per rank, with the tape replicated on every device (uploaded by each rank).
The data path has no collective; results are gathered only when the caller
wants them on one rank, and timings are reduced as the max over ranks.
"""
from __future__ import annotations

from typing import Callable, List, Tuple

import numpy as np


def shard_bounds(n_points: int, rank: int, world: int) -> Tuple[int, int]:
    """Contiguous, balanced range [lo, hi) of rank `rank` out of `world`.

    The first ``n_points % world`` ranks take one extra point, so shard sizes
    differ by at most one and the ranges tile [0, n_points) in rank order.
    """
    if world <= 0 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} out of range for world size {world}")
    base, extra = divmod(int(n_points), int(world))
    lo = rank * base + min(rank, extra)
    hi = lo + base + (1 if rank < extra else 0)
    return lo, hi


def rank_rows(global_rows: int, rank: int, world: int, seed: int, ncols: int, sampler: Callable) -> np.ndarray:
    """The rows of a seeded global batch that belong to `rank`.

    Row r of the global batch is drawn from its own stream (seed, r // 4096
    block), so every rank sees the same global batch whatever the world size.
    """
    lo, hi = shard_bounds(global_rows, rank, world)
    out = np.empty((hi - lo, ncols))
    blk = 4096
    r = lo
    while r < hi:
        b = r // blk
        rng = np.random.default_rng([seed, b])
        block = sampler(rng, (blk, ncols))
        take_lo = r - b * blk
        take_hi = min(hi - b * blk, blk)
        out[r - lo:r - lo + take_hi - take_lo] = block[take_lo:take_hi]
        r += take_hi - take_lo
    return out


def gather_rows(local: np.ndarray, group=None) -> List[np.ndarray]:
    """All ranks' result blocks, in rank order (torch.distributed object gather)."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    parts: List = [None] * world
    dist.all_gather_object(parts, local, group=group)
    return parts


def max_over_ranks(value: float, device=None, group=None) -> float:
    """The max of a per-rank scalar (a timing) over the group."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
