"""Multi-GPU mapping by replicas: every rank holds a copy of the index and maps
a contiguous share of the reads; results are merged back in input order.

Reads are independent (the reference maps them on N worker threads and only
reorders the outputs, src/shmap/mod.rs:458-636), so there is no exchange on
the data path: the only collective is the final gather of the per-rank
records, and `bench.py` does not even do that (each rank times its own share,
weak scaling).
"""
from __future__ import annotations

from typing import Callable, List, Sequence, Tuple

import numpy as np


def shard_bounds(n: int, rank: int, world: int) -> Tuple[int, int]:
    """Contiguous share [a, b) of n reads for `rank` (sizes differ by at most one)."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    q, r = divmod(n, world)
    a = rank * q + min(rank, r)
    return a, a + q + (1 if rank < r else 0)


def shard_reads(seq: np.ndarray, offs: np.ndarray, rank: int, world: int):
    """The rank's reads as (bytes, rebased offsets, global index of its first read)."""
    n = len(offs) - 1
    a, b = shard_bounds(n, rank, world)
    sub = offs[a:b + 1] - offs[a]
    return seq[offs[a]:offs[b]], sub, a


def merge_in_order(parts: Sequence[Tuple[int, np.ndarray]]) -> np.ndarray:
    """Concatenates per-rank record arrays by the global index of their first read."""
    parts = sorted(parts, key=lambda p: p[0])
    return np.concatenate([p[1] for p in parts]) if parts else np.zeros(0)


def map_replicated(map_fn: Callable[[np.ndarray, np.ndarray], np.ndarray], seq: np.ndarray, offs: np.ndarray,
                   rank: int, world: int, group=None) -> np.ndarray:
    """Maps this rank's share with `map_fn(bytes, offsets) -> records` and, with a
    torch.distributed group, gathers every rank's records on every rank in
    input order. Without a group (world 1) it is map_fn on everything."""
    s, o, first = shard_reads(seq, offs, rank, world)
    mine = map_fn(s, o)
    if world == 1:
        return mine
    import torch.distributed as dist

    got: List = [None] * world
    dist.all_gather_object(got, (first, mine), group=group)
    return merge_in_order(got)
