"""Case sharding across ranks (winds-master_b200/sharding.py): the balance of
the partition, and a world-size-2 gloo run on CPU in which each rank owns its
cases and the per-case values come back in the full case order."""
from __future__ import annotations

import importlib
import multiprocessing as mp
import os
import socket

import numpy as np


def _mod():
    return importlib.import_module("winds-master_b200.sharding")


def test_partition_covers_every_case_once_and_balances(synth):
    sh = _mod()
    cases = [synth.make_wake_case(rc, nsteps=3) for rc in synth.batch_cases(64, seed=2, steps_range=(10, 60))]
    costs = [sh.case_cost(c) for c in cases]
    for world in (1, 2, 3, 8):
        parts = sh.partition(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(cases)))
        assert sh.imbalance(costs, parts) < 1.15
    # deterministic
    assert sh.partition(costs, 4) == sh.partition(costs, 4)
    # more ranks than cases: empty ranks, no case lost
    parts = sh.partition(costs[:3], 5)
    assert sorted(i for p in parts for i in p) == [0, 1, 2]


class OracleStepper:
    """The FP64 step oracle with the lifting line and loads (oracle/kj_ref.py)
    in place of the device batch: one KJWakeRef per case of this rank."""

    def __init__(self, cases, kjs, **kw):
        import kj_ref
        import wake_ref
        self.refs = [kj_ref.KJWakeRef(wake_ref.WakeCaseRef(**{k: c[k] for k in
                                                               wake_ref.WakeCaseRef.__dataclass_fields__}),
                                      kj, integrator="pcc", relax=0.3, tol=1e-6, maxiter=60)
                     for c, kj in zip(cases, kjs)]

    def step(self, graph=True):
        for r in self.refs:
            r.step()

    def values(self):
        return np.array([[r.T, r.Q, r.P, float(r.kj_iters)] for r in self.refs])

    def close(self):
        pass


def _small_cases(n, seed=4):
    import importlib
    synth = importlib.import_module("winds-master_b200.synth")
    rcs = synth.batch_cases(n, seed=seed, steps_range=(5, 9), nodes_range=(7, 9))
    cases = [synth.make_wake_case(rc, nsteps=4) for rc in rcs]
    kjs = [synth.make_kj_case(rc, nsteps=4, t0=c["t0"]) for rc, c in zip(rcs, cases)]
    return cases, kjs


def _run_worker(rank, world, port, ncases, steps, q):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in (root, os.path.join(root, "oracle"), os.path.join(root, "tests")):
        sys.path.insert(0, p)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    import datetime
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        from test_sharding import OracleStepper, _small_cases
        sh = _mod()
        cases, kjs = _small_cases(ncases)
        run = sh.ShardedRun(cases, kjs, rank=rank, world=world, stepper=OracleStepper)
        hist = [run.step().tolist() for _ in range(steps)]
        q.put((rank, run.mine, [len(x.refs) for x in [run.local] if x is not None], hist))
        run.close()
    finally:
        dist.destroy_process_group()


def _spawn(world, ncases, steps):
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_run_worker, args=(r, world, port, ncases, steps, q))
             for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=300) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return res


def test_sharded_steps_match_a_single_rank_run():
    """Two gloo ranks each step their own cases (FP64 step oracle with the
    lifting line and loads); the gathered thrust, torque, power and iteration
    counts of every case, every step, equal those of one rank stepping all
    cases, on both ranks. A third layout puts more ranks than cases: the empty
    rank still takes part in every gather."""
    sh = _mod()
    cases, kjs = _small_cases(5)
    one = sh.ShardedRun(cases, kjs, rank=0, world=1, stepper=OracleStepper)
    want = [one.step().tolist() for _ in range(3)]
    res = _spawn(2, 5, 3)
    parts = sh.partition([sh.case_cost(c) for c in cases], 2)
    for rank, mine, local_n, hist in res:
        assert mine == parts[rank] and local_n == [len(parts[rank])]
        assert hist == want
    assert sorted(res[0][1] + res[1][1]) == list(range(5))
    few = _spawn(3, 2, 1)
    assert sum(len(m) for _, m, _, _ in few) == 2 and any(not m for _, m, _, _ in few)
    one2 = sh.ShardedRun(*_small_cases(2), rank=0, world=1, stepper=OracleStepper)
    ref2 = one2.step().tolist()
    for _, _, _, hist in few:
        assert hist == [ref2]
