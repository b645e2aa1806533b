"""Sharding across ranks (winds-master_b200/sharding.py). By case: the
balance of the partition, and a world-size-2 gloo run on CPU in which each
rank owns its cases and the per-case values come back in the full case order.
By target: the runs, the layout round trip, and gloo ranks that each evaluate
their run of one wake's targets and all-gather the field."""
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


# ---------------------------------------------------------- target sharding
def test_target_slices_cover_every_target_once():
    sh = _mod()
    for n, world in ((10, 3), (9, 3), (2, 3), (0, 2), (88803, 8)):
        sl = sh.target_slices(n, world)
        assert len(sl) == world and sl[0][0] == 0 and sl[-1][1] == n
        assert all(a[1] == b[0] for a, b in zip(sl, sl[1:]))
        sizes = [t1 - t0 for t0, t1 in sl]
        assert max(sizes) - min(sizes) <= 1


def test_target_layout_round_trip():
    """Rows of a [ns,3,m,k] column-major array, cut into runs, padded and
    assembled again, give back the array (the evaluation as the identity)."""
    import torch
    sh = _mod()
    dims = (5, 3, 4, 2)
    A = np.random.default_rng(1).normal(size=dims)
    P = torch.from_numpy(A.ravel(order="F").copy())
    for world in (1, 2, 3, 7, 50):
        blocks = []
        for r in range(world):
            ev = sh.TargetShardedEval(dims, rank=r, world=world)
            blocks.append(ev.local_block(P, lambda Pc, d, out: out.copy_(Pc)))
        out = torch.zeros_like(P)
        sh.TargetShardedEval(dims, rank=0, world=world).assemble(blocks, out)
        assert torch.equal(out, P)
    # row t is flat target t = i + ns*(j + m*b)
    ev = sh.TargetShardedEval(dims)
    rows = ev.rows(P).numpy()
    i, j, b = 3, 2, 1
    assert np.array_equal(rows[i + 5 * (j + 4 * b)], A[i, :, j, b])


def _target_case():
    import importlib
    synth = importlib.import_module("winds-master_b200.synth")
    w = synth.make_wake(synth.RotorCase(nst=7, nsteps=10, dpsi_deg=10.0, seed=9))
    fams = [synth.shed_filaments(w["dom"]) + (w["gamma_shed"], w["rc_shed"]),
            synth.trail_filaments(w["dom"]) + (w["gamma_trail"], w["rc_trail"])]
    return fams, w["dom"]


def _oracle_evaluator(fams):
    """The FP64 oracle (core/BiotSavart.m restated) on a column-major [n,3]
    run of targets, Vatistas n=2, summed over both filament families."""
    import biot_savart_ref as ref
    import torch

    def f(P_cols, dims, out_cols):
        Pn = P_cols.numpy().reshape(dims, order="F")
        u = sum(ref.biot_savart(F1, F2, Pn, g, rc, "visc2", 1000.0, "full")[0]
                for F1, F2, g, rc in fams)
        out_cols.copy_(torch.from_numpy(np.asarray(u).ravel(order="F").copy()))
    return f


def _target_worker(rank, world, port, q):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in (root, os.path.join(root, "oracle"), os.path.join(root, "tests")):
        sys.path.insert(0, p)
    import datetime
    import torch
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        from test_sharding import _oracle_evaluator, _target_case
        sh = _mod()
        fams, dom = _target_case()
        P = torch.from_numpy(np.asarray(dom).ravel(order="F").copy())
        out = torch.zeros_like(P)
        ev = sh.TargetShardedEval(dom.shape, rank=rank, world=world)
        ev(P, out, _oracle_evaluator(fams))
        q.put((rank, (ev.t0, ev.t1), out.numpy().tolist()))
    finally:
        dist.destroy_process_group()


def test_target_sharded_evaluation_on_gloo_ranks():
    """Two and three gloo ranks each evaluate their run of one wake's targets
    (FP64 oracle) and all-gather: every rank holds exactly the field of one
    evaluation of all targets."""
    import torch
    sh = _mod()
    fams, dom = _target_case()
    P = torch.from_numpy(np.asarray(dom).ravel(order="F").copy())
    want = torch.zeros_like(P)
    _oracle_evaluator(fams)(P, dom.shape, want)
    for world in (2, 3):
        with socket.socket() as s:
            s.bind(("127.0.0.1", 0))
            port = s.getsockname()[1]
        ctx = mp.get_context("spawn")
        q = ctx.Queue()
        procs = [ctx.Process(target=_target_worker, args=(r, world, port, q)) for r in range(world)]
        for p in procs:
            p.start()
        res = sorted(q.get(timeout=300) for _ in range(world))
        for p in procs:
            p.join(timeout=60)
            assert p.exitcode == 0
        assert [r[1] for r in res] == sh.target_slices(P.numel() // 3, world)
        for _, _, got in res:
            assert np.array_equal(np.array(got), want.numpy())
