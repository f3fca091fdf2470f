"""Sharding of independent Monte-Carlo work over ranks (one process per GPU).

Instances, solve requests and SA restarts are independent units, so the
multi-GPU form of the hot path partitions them across ranks with no
collective on the data path; only a final gather of results crosses ranks.
`partition` is a longest-processing-time-first assignment by cost (flips),
deterministic so every rank computes the same plan without communicating.
"""
from __future__ import annotations

import heapq
from typing import Sequence


def partition(costs: Sequence[float], world: int) -> list[list[int]]:
    """Unit indices per rank, balancing the summed cost (LPT greedy)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda k: (-costs[k], k))
    heap = [(0.0, r) for r in range(world)]
    out: list[list[int]] = [[] for _ in range(world)]
    for k in order:
        load, r = heapq.heappop(heap)
        out[r].append(k)
        heapq.heappush(heap, (load + float(costs[k]), r))
    return [sorted(x) for x in out]


def restart_seeds(base_seed: int, rank: int, per_rank: int) -> list[int]:
    """Disjoint seeds for the SA restarts of one rank."""
    return [base_seed + rank * per_rank + k for k in range(per_rank)]


def gather(obj, world: int):
    """All-gather of a picklable per-rank result (torch.distributed object
    collective); identity when running on one rank."""
    if world == 1:
        return [obj]
    import torch.distributed as dist
    out = [None] * world
    dist.all_gather_object(out, obj)
    return out
