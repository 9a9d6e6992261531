"""Multi-GPU sharding of walk batches: one process per GPU.

Walks are independent, so ranks take disjoint shards and run them with no
collective on the data path.  The only exchange is the final top-k: each rank
contributes its local best (delta, global walk index) pairs and every rank
ends up with the same global top-k, ordered by delta (highest first) and
then by lower walk index -- the same order the device top-k uses.
"""

from __future__ import annotations

from typing import List, Sequence, Tuple

__all__ = ["shard_range", "merge_topk", "global_topk"]


def shard_range(n: int, rank: int, world: int) -> Tuple[int, int]:
    """Contiguous [start, stop) share of ``n`` walks for ``rank``."""
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def _key(item):
    delta, idx = item
    # NaN ranks last, then higher delta first, then lower index
    nan = delta != delta
    return (nan, -delta if not nan else 0.0, idx)


def merge_topk(parts: Sequence[Sequence[Tuple[float, int]]], k: int) -> List[Tuple[float, int]]:
    """Merge per-rank (delta, global index) lists into the global top-k."""
    allv = [tuple(x) for p in parts for x in p]
    return sorted(allv, key=_key)[:k]


def global_topk(local: Sequence[Tuple[float, int]], k: int, group=None) -> List[Tuple[float, int]]:
    """All-gather every rank's local top-k and merge (torch.distributed)."""
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return merge_topk([local], k)
    world = dist.get_world_size(group)
    parts: List = [None] * world
    dist.all_gather_object(parts, [(float(d), int(i)) for d, i in local], group=group)
    return merge_topk(parts, k)
