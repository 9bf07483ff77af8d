"""Rate-set shards across ranks (one process per GPU).

A solve is one (network, rate set, initial distribution) triple.  Once a network's
symbolic data exists, the solves are independent, so a sweep is split across ranks
by contiguous slices of rate sets.  Each rank builds the network's symbolic data
itself, and no data-path collective is involved: the only collective is the
max-over-ranks reduction of timings and error figures.  The reference has no
multi-GPU code; this is the natural partition of its batched use (many rate sets
per network).

Weak scaling: the global sweep of a W-rank run is W x B rate sets (B per rank).
The first B are the given sweep (the held-out rate sets of the benchmark); the
rest are further seeded draws of the same distribution, identical on every rank.
Rank r solves the slice ``shard_bounds(W * B, r, W)`` of it, so at W = 1 the run
is exactly the given sweep, and every global rate set is solved exactly once.
"""
from __future__ import annotations

from typing import Callable, Tuple

import numpy as np


def shard_bounds(total: int, rank: int, world: int) -> Tuple[int, int]:
    """[begin, end) of rank's contiguous slice of ``total`` items; sizes differ by at most one."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world of {world}")
    if total < 0:
        raise ValueError("negative total")
    base, extra = divmod(total, world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def global_sweep(first: np.ndarray, world: int, draw: Callable[[int, int], np.ndarray]) -> np.ndarray:
    """The W x B global rate-set sweep: ``first`` (B x 2n) then ``draw(seed, B)`` for
    seeds 1 .. W-1 (each B x 2n), concatenated."""
    if world < 1:
        raise ValueError(f"world of {world}")
    parts = [np.asarray(first)]
    for r in range(1, world):
        extra = np.asarray(draw(r, len(first)))
        if extra.shape != parts[0].shape:
            raise ValueError(f"draw returned {extra.shape}, expected {parts[0].shape}")
        parts.append(extra)
    return np.concatenate(parts, axis=0)


def rank_rate_sets(first: np.ndarray, rank: int, world: int,
                   draw: Callable[[int, int], np.ndarray]) -> Tuple[np.ndarray, Tuple[int, int]]:
    """This rank's contiguous slice of the global sweep and its [begin, end) bounds."""
    sweep = global_sweep(first, world, draw)
    b, e = shard_bounds(len(sweep), rank, world)
    return np.ascontiguousarray(sweep[b:e]), (b, e)


def max_over_ranks(values, world: int, device=None):
    """Element-wise max of a list of per-rank floats over all ranks (the values
    themselves without a process group).  ``device`` is the rank's CUDA device
    under NCCL, None under gloo."""
    vals = [float(v) for v in values]
    if world <= 1:
        return vals
    import torch
    import torch.distributed as dist

    t = torch.tensor(vals, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.cpu()]
