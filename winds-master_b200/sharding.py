"""Case sharding across GPUs (one process per GPU).

Every rotor case is independent: its wake nodes see only its own filaments.
So a multi-GPU run splits the list of cases, each rank steps its own batch
with no collective on the data path, and only per-step scalars (loads,
iteration counts) cross ranks, gathered on the host after the step. The
split balances the per-step direct-sum work: greedy longest-processing-time
assignment of each case's interactions per evaluation (nodes x filaments
plus the lifting line), heaviest first, ties to the lowest rank.
"""
from __future__ import annotations

import heapq

import numpy as np


def case_cost(case: dict) -> int:
    """Interactions of one evaluation of a case (wake nodes + lifting-line
    points against shed + trailing filaments)."""
    nst, na, nb = int(case["nst"]), int(case["na"]), int(case["nb"])
    nodes = nst * na * nb
    fil = ((nst - 1) * na + nst * (na - 1)) * nb
    return (nodes + (nst - 1) * nb) * fil


def partition(costs, world: int):
    """Case indices of every rank: longest processing time first. Returns a
    list of ``world`` sorted index lists (deterministic)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0, r) for r in range(world)]
    out = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(x) for x in out]


def imbalance(costs, parts) -> float:
    """max rank load / mean rank load (1.0 is perfect)."""
    loads = [sum(costs[i] for i in p) for p in parts]
    mean = sum(loads) / max(len(loads), 1)
    return max(loads) / mean if mean > 0 else 1.0


def gather_case_values(values_local, parts, rank: int, world: int, group=None):
    """Reassembles per-case values (one row per case of this rank, in the
    order of ``parts[rank]``) into the full case order on every rank, through
    torch.distributed all_gather_object (host data, after the step)."""
    import torch.distributed as dist
    local = np.asarray(values_local)
    if world == 1:
        return local
    got = [None] * world
    dist.all_gather_object(got, (rank, local.tolist()), group=group)
    n = sum(len(p) for p in parts)
    first = np.asarray(got[0][1])
    out = np.zeros((n,) + first.shape[1:], dtype=first.dtype if first.size else np.float64)
    for r, vals in got:
        for j, i in enumerate(parts[r]):
            out[i] = vals[j]
    return out
