"""Work distribution of (channel, energy) solves over ranks (one process per GPU).

The solves are independent (the reference shards 3N channels over processes,
CPP/main.cpp:168-170); there is no collective on the data path.  The unit of
work is a (channel, on-shell energy) item of LU cost ~ n^3; the energies of one
channel that a rank owns are solved in one call (one A build, their matrices
factored together), so items are grouped per channel in runs of up to
`group` energies before the longest-processing-time assignment.  Ranks only
exchange scalars (the step time, for max-over-ranks timing) and, at the end,
the small U arrays, which rank 0 assembles in the reference's layout
U[d' nd nE + d nE + j] per channel (CPP/solve_faddeev.cpp:424).
"""
from __future__ import annotations

import heapq

import numpy as np


def lpt_partition(weights, world):
    """Greedy longest-processing-time assignment of items to `world` ranks.
    Returns one list of item indices per rank; the heaviest items go first
    (ties in item order), each to the least-loaded rank (ties to the lowest)."""
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    out = [[] for _ in range(world)]
    for i in sorted(range(len(weights)), key=lambda i: (-weights[i], i)):
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + weights[i], r))
    return [sorted(x) for x in out]


def channel_weights(dense_dims, n_energies=1):
    """LU cost of a channel ~ n^3 per energy."""
    return [n_energies * float(n) ** 3 for n in dense_dims]


def scan_items(dense_dims, n_energies, group=2):
    """(channel, energies) items: each channel's on-shell energies in runs of
    up to `group` consecutive indices, weighted by n^3 per energy."""
    items, weights = [], []
    for c, n in enumerate(dense_dims):
        for j0 in range(0, n_energies, group):
            js = list(range(j0, min(n_energies, j0 + group)))
            items.append((c, js))
            weights.append(len(js) * float(n) ** 3)
    return items, weights


def plan(dense_dims, n_energies, world, group=2):
    """Per rank, {channel: [energy indices]} of the items it owns."""
    items, weights = scan_items(dense_dims, n_energies, group)
    out = []
    for part in lpt_partition(weights, world):
        mine = {}
        for i in part:
            c, js = items[i]
            mine.setdefault(c, []).extend(js)
        out.append({c: sorted(js) for c, js in sorted(mine.items())})
    return out


def rank_load(rank_plan, dense_dims):
    return sum(len(js) * float(dense_dims[c]) ** 3 for c, js in rank_plan.items())


def run_plan(rank_plan, solve):
    """Solve this rank's items: solve(channel, energy_indices) -> U of those
    energies in the layout [d'][d][s].  Returns {channel: (energies, U)}."""
    return {c: (list(js), np.asarray(solve(c, js))) for c, js in rank_plan.items()}


def assemble_U(gathered, n_deuteron, n_energies):
    """Rank 0: merge every rank's {channel: (energies, U[d'][d][s])} into one
    array per channel in the reference's layout U[d' nd nE + d nE + j].
    Every (channel, energy) must come from exactly one rank."""
    out = {c: np.zeros(nd * nd * n_energies, dtype=np.complex128) for c, nd in enumerate(n_deuteron)}
    seen = {c: np.zeros(n_energies, dtype=int) for c in out}
    for part in gathered:
        for c, (js, U) in part.items():
            nd = n_deuteron[c]
            Us = np.asarray(U).reshape(nd, nd, len(js))
            full = out[c].reshape(nd, nd, n_energies)
            for s, j in enumerate(js):
                full[:, :, j] = Us[:, :, s]
                seen[c][j] += 1
    for c, cnt in seen.items():
        if n_deuteron[c] and not np.all(cnt == 1):
            raise ValueError(f"channel {c}: energies solved {cnt.tolist()} times")
    return out


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
