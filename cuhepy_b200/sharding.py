"""Sharding across GPUs of one node (one process per GPU, torch.distributed).

Both paths shard without a data-path collective: Paillier ciphertexts are
independent items, and a BFV search's response groups (``padded``
consecutive tiles merged into one response, ``bfv_server.h:15-45`` of the
reference) are independent of one another.  A rank owns a contiguous shard;
the only collectives are a barrier before timing and the maximum of the
elapsed times over ranks.  The host gathers per-shard results in rank order,
which reproduces the unsharded order.
"""

from __future__ import annotations

from typing import Any


def shard_bounds(total: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous, balanced [lo, hi) share of `total` items for `rank`."""
    if world < 1 or not 0 <= rank < world or total < 0:
        raise ValueError("invalid shard request")
    base, extra = divmod(int(total), int(world))
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def group_shard_bounds(tiles: int, padded: int, rank: int, world: int) -> tuple[int, int]:
    """Tile range [lo, hi) of `rank` made of whole response groups of
    `padded` tiles (the last group may be short), so each rank's responses
    are exactly the unsharded responses of its groups."""
    if padded < 1:
        raise ValueError("padded must be positive")
    groups = (int(tiles) + padded - 1) // padded
    g_lo, g_hi = shard_bounds(groups, rank, world)
    return min(tiles, g_lo * padded), min(tiles, g_hi * padded)


def max_over_ranks(value: float, dist: Any = None, device: Any = "cpu") -> float:
    """Maximum of `value` over all ranks (the job's elapsed time); `value`
    itself when no process group is running."""
    if dist is None or not dist.is_available() or not dist.is_initialized():
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_in_rank_order(local: list, dist: Any = None) -> list:
    """Concatenate every rank's list of results in rank order (host objects)."""
    if dist is None or not dist.is_available() or not dist.is_initialized():
        return list(local)
    parts: list = [None] * dist.get_world_size()
    dist.all_gather_object(parts, list(local))
    return [item for part in parts for item in part]
