"""Case sharding across GPUs (one process per GPU).

Every rotor case is independent: its wake nodes see only its own filaments.
So a multi-GPU run splits the list of cases, each rank steps its own batch
with no collective on the data path, and only per-step scalars (loads,
iteration counts) cross ranks, gathered on the host after the step. The
split balances the per-step direct-sum work: greedy longest-processing-time
assignment of each case's interactions per evaluation (nodes x filaments
plus the lifting line), heaviest first, ties to the lowest rank.

``ShardedRun`` is the driver: every rank builds the batch of its own cases
(``partition(...)[rank]``) through a stepper factory -- ``BatchStepper`` (the
device engine, ``wake.WakeBatch``) by default -- steps it, and after every
step gathers thrust, torque, power and iteration counts of all cases in case
order on every rank. A rank without cases (more ranks than cases) steps
nothing and still joins every gather.
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
    dist.all_gather_object(got, (rank, local.shape[1:], local.tolist()), group=group)
    n = sum(len(p) for p in parts)
    tail = next((shp for _, shp, v in got if len(v)), local.shape[1:])
    dtype = next((np.asarray(v).dtype for _, _, v in got if len(v)), np.float64)
    out = np.zeros((n,) + tuple(tail), dtype=dtype)
    for r, _, vals in got:
        for j, i in enumerate(parts[r]):
            out[i] = vals[j]
    return out


class BatchStepper:
    """The device engine for one rank's cases: a ``wake.WakeBatch`` (with the
    lifting lines when ``kjs`` is given). ``step`` advances one step;
    ``values`` returns per-case rows (thrust, torque, power, iterations)."""

    def __init__(self, cases, kjs=None, kj_params=None, **batch_kw):
        from .wake import WakeBatch
        self.b = WakeBatch(cases, **batch_kw)
        self.kj = kjs is not None
        if self.kj:
            self.b.set_kj(kjs, **(kj_params or {}))
        self.n = len(cases)

    def step(self, graph=True):
        self.b.step(1, graph=graph)

    def values(self):
        if not self.kj:
            return np.zeros((self.n, 4))
        T, Q, P = self.b.loads()
        it = self.b.kj_stats()[0]
        return np.stack([T, Q, P, it.astype(np.float64)], 1)

    def step_ms(self):
        return self.b.stats()[0]

    def close(self):
        self.b.close()


class ShardedRun:
    """Steps ``cases`` (wake-case dicts, with ``kjs`` lifting lines when given)
    split over ``world`` ranks; this process is ``rank``. ``stepper`` builds
    the local stepper from (cases, kjs, **kw); after every ``step`` the
    per-case rows of ``values()`` of all ranks are in ``history`` (one
    [ncases, columns] array per step, case order), the same on every rank."""

    def __init__(self, cases, kjs=None, rank=0, world=1, stepper=BatchStepper, group=None,
                 **kw):
        self.rank, self.world, self.group = rank, world, group
        self.parts = partition([case_cost(c) for c in cases], world)
        self.mine = self.parts[rank]
        self.ncases = len(cases)
        self.local = None
        if self.mine:
            self.local = stepper([cases[i] for i in self.mine],
                                 None if kjs is None else [kjs[i] for i in self.mine], **kw)
        self.history = []

    def step(self, n=1, graph=True):
        for _ in range(n):
            if self.local is not None:
                self.local.step(graph=graph)
                vals = self.local.values()
            else:
                vals = np.zeros((0, 4))
            self.history.append(gather_case_values(vals, self.parts, self.rank, self.world, self.group))
        return self.history[-1]

    def close(self):
        if self.local is not None:
            self.local.close()
            self.local = None
