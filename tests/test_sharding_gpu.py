"""Target sharding of one evaluation on the GPU (sharding.TargetShardedEval
with the engine's device evaluation). Ranks are emulated in one process by
evaluating each rank's run in turn (nothing waits on another rank); the
collective path runs through a one-rank NCCL process group."""
from __future__ import annotations

import importlib
import socket

import numpy as np
import pytest

from conftest import per_target_rel

pytestmark = pytest.mark.gpu


def _setup(wb, synth):
    import torch
    w = synth.make_wake(synth.RotorCase(nst=17, nsteps=60, dpsi_deg=10.0, seed=31))
    fams = [synth.shed_filaments(w["dom"]) + (w["gamma_shed"], w["rc_shed"]),
            synth.trail_filaments(w["dom"]) + (w["gamma_trail"], w["rc_trail"])]
    dev = lambda a: torch.from_numpy(np.asarray(a).ravel(order="F").copy()).cuda()
    dfams = [(dev(F1), dev(F2), dev(g), dev(rc), F1.shape) for F1, F2, g, rc in fams]
    return dfams, dev(w["dom"]), w["dom"].shape


def test_emulated_ranks_assemble_the_full_field(wb, synth):
    """Each of 1, 3 and 8 emulated ranks evaluates its run of targets with the
    engine; the assembled field equals one evaluation of all targets (FP32c
    1e-5, FP64 1e-12 per-target relative)."""
    import torch
    sh = importlib.import_module("winds-master_b200.sharding")
    dfams, P, dims = _setup(wb, synth)
    for prec, tol in (("f32c", 1e-5), ("f64", 1e-12)):
        want = torch.zeros_like(P)
        wb.eval_device(dfams, (P, dims), wb.bs.CORE_VATISTAS, 2.0, 1000.0, want, prec)
        wb.sync()
        ev = sh.device_evaluator(dfams, wb.bs.CORE_VATISTAS, 2.0, 1000.0, prec)
        for world in (1, 3, 8):
            parts = [sh.TargetShardedEval(dims, rank=r, world=world) for r in range(world)]
            blocks = [p.local_block(P, ev) for p in parts]
            wb.sync()
            out = torch.full_like(P, float("nan"))
            parts[0].assemble(blocks, out)
            u = out.cpu().numpy().reshape(dims, order="F")
            u_ref = want.cpu().numpy().reshape(dims, order="F")
            assert np.all(np.isfinite(u))
            assert per_target_rel(u, u_ref) < tol, (prec, world)


def test_nccl_all_gather_path_on_one_rank(wb, synth):
    """The collective path (NCCL all-gather of the padded blocks) on a
    one-rank process group gives the same bits as the path without one."""
    import datetime
    import torch
    import torch.distributed as dist
    sh = importlib.import_module("winds-master_b200.sharding")
    dfams, P, dims = _setup(wb, synth)
    ev = sh.device_evaluator(dfams, wb.bs.CORE_VATISTAS, 2.0, 1000.0, "f32c")
    plain = torch.zeros_like(P)
    sh.TargetShardedEval(dims)(P, plain, ev)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        out = torch.zeros_like(P)
        sh.TargetShardedEval(dims, rank=0, world=1, group=dist.group.WORLD)(P, out, ev)
        torch.cuda.synchronize()
    finally:
        dist.destroy_process_group()
    assert torch.equal(out, plain)
