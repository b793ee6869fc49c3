"""Sharding of independent models across ranks (one process per GPU).

A batch of independent systems (e.g. 512 plates) needs no exchange while it is
factored and solved: each rank takes a share of the models, balanced by the flop
estimate of their symbolic analyses (``Symbolic::work``, src/sparse.rs:236-238),
and factors its share as one batched factorization. The only collective is the
final gather of the solutions (or nothing, when each rank keeps its own). A single
model does not shard: ranks run replicas.
"""
from __future__ import annotations

import heapq

import numpy as np


def partition(work, world: int) -> list[list[int]]:
    """Greedy longest-processing-time split of models (given their work) into
    ``world`` shares; each share keeps the models in their original order."""
    work = [float(w) for w in work]
    order = sorted(range(len(work)), key=lambda i: (-work[i], i))
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    shares = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        shares[r].append(i)
        heapq.heappush(heap, (load + work[i], r))
    return [sorted(s) for s in shares]


def imbalance(work, shares) -> float:
    """Largest share's work over the mean share's work (1.0 = perfect)."""
    loads = [sum(work[i] for i in s) for s in shares]
    mean = sum(loads) / max(len(loads), 1)
    return max(loads) / mean if mean > 0 else 1.0


def gather_solutions(local: dict, world: int, dist) -> dict:
    """All ranks' {model index: solution} merged on every rank (torch.distributed
    object all-gather; gloo or NCCL process group)."""
    if world == 1:
        return dict(local)
    parts = [None] * world
    dist.all_gather_object(parts, {int(k): np.asarray(v) for k, v in local.items()})
    out = {}
    for p in parts:
        out.update(p)
    return out
