"""Sharding independent solves across ranks (one process per GPU).

Poisson solves of different images (and channels) are independent, so N GPUs
scale by giving each rank its own share of the images: no collective is needed
on the data path. The split is greedy longest-processing-time on an estimated
cost (interior pixels x channels x expected sweeps), ties broken by image
index, so every rank computes the same plan without communicating. Results are
gathered to rank 0 in image order with a single object gather -- the only
collective, and only for the host-side report.
"""
from __future__ import annotations

import heapq
from typing import Callable, Sequence


def estimate_cost(width: int, height: int, channels: int, interior: int | None = None,
                  sweeps: float = 1.0) -> float:
    """Relative cost of one image: interior cells x channels x expected sweeps.
    For multigrid-preconditioned CG, whose iteration count hardly changes with
    the region and whose kernels pass over every cell of the image, leave
    `interior` and `sweeps` at their defaults: pixels x channels."""
    n = interior if interior is not None else width * height
    return float(n) * float(channels) * float(sweeps)


def partition(costs: Sequence[float], world_size: int) -> list[list[int]]:
    """Greedy LPT: images in decreasing cost (then index) go to the least loaded
    rank (then lowest rank). Deterministic; returns each rank's image indices
    in increasing order."""
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(world_size)]
    heapq.heapify(heap)
    shares: list[list[int]] = [[] for _ in range(world_size)]
    for i in order:
        load, r = heapq.heappop(heap)
        shares[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(s) for s in shares]


def run_sharded(items: Sequence, costs: Sequence[float], solve: Callable, rank: int,
                world_size: int, group=None):
    """Solve this rank's share with `solve(item)` and gather every result to
    rank 0 in item order. Returns the full result list on rank 0, None elsewhere.
    Uses torch.distributed when world_size > 1 (any backend)."""
    share = partition(costs, world_size)[rank]
    mine = {i: solve(items[i]) for i in share}
    if world_size == 1:
        return [mine[i] for i in range(len(items))]
    import torch.distributed as dist
    gathered = [None] * world_size if rank == 0 else None
    dist.gather_object(mine, gathered, dst=0, group=group)
    if rank != 0:
        return None
    merged = {}
    for part in gathered:
        merged.update(part)
    return [merged[i] for i in range(len(items))]
