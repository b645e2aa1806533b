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

One wake can also be split by target (``TargetShardedEval``): every rank
holds all filaments and all targets, evaluates the induced velocity at a
contiguous run of the targets (the WInDS flat order span + ns*(age +
na*blade), so a run is a band of wake ages, compact in space) and one
all-gather of the velocities (NCCL on GPUs) gives every rank the whole field
for its identical convection step. The exchange is 24 bytes per target.
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


# ------------------------------------------------------------ target sharding
def target_slices(n_targets: int, world: int):
    """``[t0, t1)`` of every rank: contiguous runs of the flat target order,
    sizes differing by at most one (the first ``n % world`` ranks one more)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    base, extra = divmod(int(n_targets), world)
    out, t0 = [], 0
    for r in range(world):
        t1 = t0 + base + (1 if r < extra else 0)
        out.append((t0, t1))
        t0 = t1
    return out


def _dims4(dims):
    d = [int(x) for x in dims]
    while len(d) < 4:
        d.append(1)
    if len(d) != 4 or d[1] != 3:
        raise ValueError(f"target dims must be [n,3,m,k], got {dims}")
    return d


def device_evaluator(families, core, d, co, precision="f32c", stream=None):
    """The engine's device evaluation (``bs.eval_device``) as the callable
    ``TargetShardedEval`` takes: ``f(P_cols, dims, out_cols)`` with torch CUDA
    tensors, ``P_cols`` and ``out_cols`` column-major ``[n,3]``. It runs on
    ``stream`` (a CUDA stream handle), by default on torch's current stream at
    the time of the call, the stream the tensor operations around it (the
    target gather, the padding copy, the all-gather) are ordered on."""
    from .bs import eval_device

    def f(P_cols, dims, out_cols):
        import torch
        if stream is not None:
            eval_device(families, (P_cols, dims), core, d, co, out_cols, precision, stream=stream)
            return
        cur = torch.cuda.current_stream()
        if cur.cuda_stream != 0:
            eval_device(families, (P_cols, dims), core, d, co, out_cols, precision,
                        stream=cur.cuda_stream)
            return
        # torch's legacy default stream has handle 0, which the engine reads as
        # "its own stream": run on a side stream ordered after and before it
        side = _side_stream(cur.device)
        side.wait_stream(cur)
        eval_device(families, (P_cols, dims), core, d, co, out_cols, precision,
                    stream=side.cuda_stream)
        cur.wait_stream(side)
    return f


_SIDE = {}


def _side_stream(device):
    import torch
    if device not in _SIDE:
        _SIDE[device] = torch.cuda.Stream(device=device)
    return _SIDE[device]


class TargetShardedEval:
    """One induced-velocity evaluation of a ``[ns,3,m,k]`` target array split
    over ``world`` ranks by target; this process is ``rank``.

    ``__call__(P, out, evaluate)``: ``P`` and ``out`` are flat float64 torch
    tensors holding the column-major ``[ns,3,m,k]`` targets and velocities (the
    same ``P`` on every rank); ``evaluate(P_cols, dims, out_cols)`` computes
    this rank's run (``device_evaluator`` for the engine). The runs are padded
    to one size and exchanged with a single all-gather of ``[3, n_max]``
    blocks on ``group`` (the default group when None; with ``world`` 1 and
    no group, no collective); every rank then holds the whole field in ``out``.
    Every rank makes the same collective call, also a rank whose run is
    empty (more ranks than targets)."""

    def __init__(self, pdims, rank=0, world=1, group=None):
        self.dims = _dims4(pdims)
        ns, _, m, k = self.dims
        self.n = ns * m * k
        self.rank, self.world, self.group = rank, world, group
        self.slices = target_slices(self.n, world)
        self.t0, self.t1 = self.slices[rank]
        self.n_max = max(t1 - t0 for t0, t1 in self.slices)

    def rows(self, P):
        """The targets as an ``[n,3]`` view, row t = flat target t."""
        ns, _, m, k = self.dims
        return P.view(k, m, 3, ns).permute(0, 1, 3, 2).reshape(self.n, 3)

    def local_targets(self, P):
        """This rank's run as a column-major ``[n_r,3]`` tensor (a copy)."""
        return self.rows(P)[self.t0:self.t1].t().contiguous().view(-1)

    def assemble(self, blocks, out):
        """Writes the gathered ``[3, n_max]`` blocks (rank order) into ``out``
        in the ``[ns,3,m,k]`` layout."""
        import torch
        ns, _, m, k = self.dims
        full = torch.cat([b.view(3, self.n_max)[:, :t1 - t0]
                          for b, (t0, t1) in zip(blocks, self.slices)], dim=1)
        out.view(k, m, 3, ns).copy_(full.view(3, k, m, ns).permute(1, 2, 0, 3))
        return out

    def local_block(self, P, evaluate):
        """This rank's velocities as a zero-padded ``[3, n_max]`` block."""
        import torch
        nr = self.t1 - self.t0
        blk = torch.zeros((3, self.n_max), dtype=P.dtype, device=P.device)
        if nr > 0:
            res = torch.empty(3 * nr, dtype=P.dtype, device=P.device)
            evaluate(self.local_targets(P), (nr, 3, 1, 1), res)
            blk[:, :nr].copy_(res.view(3, nr))
        return blk

    def __call__(self, P, out, evaluate):
        blk = self.local_block(P, evaluate)
        if self.world == 1 and self.group is None:  # one rank, no process group
            blocks = [blk]
        else:
            import torch
            import torch.distributed as dist
            blocks = [torch.empty_like(blk) for _ in range(self.world)]
            dist.all_gather(blocks, blk, group=self.group)
        return self.assemble(blocks, out)
