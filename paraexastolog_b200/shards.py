"""Rate-set shards across ranks (one process per GPU).

A solve is one (network, rate set, initial distribution) triple.  Once a network's
symbolic data exists, the solves are independent, so a sweep is split across ranks
by contiguous slices of rate sets.  Each rank builds the network's symbolic data
itself, and no data-path collective is involved.  The host reduces step timings
as the max over ranks.  The reference has no multi-GPU code; this is the natural
partition of its batched use (many rate sets per network).
"""
from __future__ import annotations

from typing import Tuple


def shard_bounds(total: int, rank: int, world: int) -> Tuple[int, int]:
    """[begin, end) of rank's contiguous slice of ``total`` items; sizes differ by at most one."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world of {world}")
    if total < 0:
        raise ValueError("negative total")
    base, extra = divmod(total, world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def max_over_ranks(value: float, world: int, device=None) -> float:
    """Max of a per-rank timing over all ranks (identity without a process group)."""
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
