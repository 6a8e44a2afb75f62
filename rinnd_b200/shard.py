"""Multi-GPU placement of the batched form: independent indices are spread over
ranks (one process per GPU) by greedy longest-processing-time assignment on an
estimated cost n * d * k; every rank computes the same assignment from the same
sizes, builds its share with rinnd_build_many on its own GPU, and no data
crosses ranks (the indices are independent).  Results stay on the rank that
built them; `gather_counts` is the only collective, for reporting.
"""
from __future__ import annotations

import heapq
from typing import Sequence


def build_cost(n: int, d: int, k: int) -> float:
    """Estimated build work of one index (points x dimension x neighbors)."""
    return float(n) * float(max(d, 1)) * float(max(k, 1))


def assign_longest_first(costs: Sequence[float], world_size: int) -> list[list[int]]:
    """Greedy LPT: items in decreasing cost (ties by index) each go to the rank
    with the least assigned cost (ties by rank).  Deterministic, so all ranks
    agree without communicating.  Returns the item indices of every rank, each
    list in decreasing cost order."""
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(world_size)]
    out: list[list[int]] = [[] for _ in range(world_size)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return out


def my_share(costs: Sequence[float], rank: int, world_size: int) -> list[int]:
    return assign_longest_first(costs, world_size)[rank]


def gather_counts(local_items: int, local_points: int) -> tuple[int, int]:
    """Sum of (items, points) built over all ranks (torch.distributed, any backend)."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([local_items, local_points], dtype=torch.int64)
    if dist.is_available() and dist.is_initialized():
        if dist.get_backend() == "nccl":
            t = t.cuda()
        dist.all_reduce(t)
    return int(t[0]), int(t[1])
