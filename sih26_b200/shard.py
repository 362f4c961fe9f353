"""Sharding independent LPs over ranks (one process per GPU).

A batch of independent LPs has no data exchange between instances, so several GPUs split the
batch and run with no collective on the data path: each rank solves its own shard on its own
GPU and the answers are gathered on the host at the end. Shards are balanced by nonzeros
(each iteration streams every nonzero of an LP twice), greedily, largest LP first.
"""
from __future__ import annotations

import heapq
from typing import List, Sequence


def shard_by_nnz(nnz: Sequence[int], world: int) -> List[List[int]]:
    """Indices of the LPs for each of `world` ranks: LPs in decreasing nonzero order, each to
    the rank with the least nonzeros so far (ties to the lower rank). Deterministic; every
    index lands in exactly one shard; each shard lists its indices in increasing order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(nnz)), key=lambda k: (-int(nnz[k]), k))
    heap = [(0, r) for r in range(world)]
    shards: List[List[int]] = [[] for _ in range(world)]
    for k in order:
        load, r = heapq.heappop(heap)
        shards[r].append(k)
        heapq.heappush(heap, (load + int(nnz[k]), r))
    return [sorted(s) for s in shards]


def gather_by_index(local: dict, dist=None) -> dict:
    """Merges {index: value} dicts of every rank (all_gather_object over the default process
    group when `dist` is given); every rank gets the whole mapping."""
    if dist is None:
        return dict(local)
    parts = [None] * dist.get_world_size()
    dist.all_gather_object(parts, local)
    out = {}
    for p in parts:
        for k, v in p.items():
            if k in out:
                raise ValueError(f"index {k} came back from two ranks")
            out[k] = v
    return out
