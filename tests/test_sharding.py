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


def _worker(rank, world, port, costs, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    import datetime
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        sh = _mod()
        parts = sh.partition(costs, world)
        # each rank "steps" its own cases: per-case values computed locally
        local = [[float(i), float(costs[i]) * 2.0] for i in parts[rank]]
        full = sh.gather_case_values(local, parts, rank, world)
        q.put((rank, full.tolist()))
    finally:
        dist.destroy_process_group()


def test_gloo_two_ranks_gather_in_case_order():
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    costs = [5, 3, 9, 1, 7, 2, 8]
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, costs, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want = [[float(i), 2.0 * c] for i, c in enumerate(costs)]
    for _, full in res:
        assert full == want
