"""Work distribution of (channel, energy) solves over ranks (one process per GPU).

The solves are independent (the reference shards 3N channels over processes,
CPP/main.cpp:168-170); there is no collective on the data path.  Ranks only
exchange scalars (the step time, for max-over-ranks timing) and, at the end,
the small U arrays for rank 0.
"""
from __future__ import annotations

import heapq


def lpt_partition(weights, world):
    """Greedy longest-processing-time assignment of items to `world` ranks.
    Returns one list of item indices per rank; the heaviest items go first."""
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    out = [[] for _ in range(world)]
    for i in sorted(range(len(weights)), key=lambda i: -weights[i]):
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + weights[i], r))
    return [sorted(x) for x in out]


def channel_weights(dense_dims, n_energies=1):
    """LU cost of a channel ~ n^3 per energy."""
    return [n_energies * float(n) ** 3 for n in dense_dims]


def rank_lab_energies(base_mev, rank, spacing_mev=6.0):
    """Energy-scan replicas: rank r solves its own lab energy."""
    return base_mev + spacing_mev * rank


def max_over_ranks(dist, value, device=None):
    if dist is None or not dist.is_initialized():
        return value
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_to_rank0(dist, obj):
    """Collect a small picklable object (e.g. {channel: U}) from every rank on rank 0."""
    if dist is None or not dist.is_initialized():
        return [obj]
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, obj)
    return out if dist.get_rank() == 0 else None
