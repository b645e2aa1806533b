"""GPU test of winds_bs_eval_device_noalloc, the evaluation for callers that
cannot allocate device memory (a host that owns all device memory through its
own pool, or a per-step solver loop that cannot afford cudaMalloc's device
synchronisation). It must give winds_bs_eval_device's answer, within the FP32
path's 1e-5 tolerance (1e-12 on the FP64 path), on two calls in a row that
share its static scratch, up to exactly its target limit, without changing
the device's free memory. The file name makes pytest collect it last."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import per_target_rel

pytestmark = pytest.mark.gpu

F32C_TOL = 1e-5
F64_TOL = 1e-12
MAX_TARGETS = 65536  # WINDS_BS_NOALLOC_MAX_TARGETS


def _device_inputs(wb, synth, case):
    import torch
    w = synth.make_wake(case)
    fams = [synth.shed_filaments(w["dom"]) + (w["gamma_shed"], w["rc_shed"]),
            synth.trail_filaments(w["dom"]) + (w["gamma_trail"], w["rc_trail"])]
    dev = lambda a: torch.from_numpy(np.asarray(a).ravel(order="F").copy()).cuda()
    dfams = [(dev(F1), dev(F2), dev(g), dev(rc), F1.shape) for F1, F2, g, rc in fams]
    P = w["dom"]
    return dfams, dev(P), P.shape


def _noalloc(wb, dfams, dP, pshape, out, core, d, stream, prec="f32c"):
    L = wb.lib()
    fam = (wb.bs.Family * len(dfams))()
    for k, (F1, F2, g, rc, dims) in enumerate(dfams):
        fam[k].F1, fam[k].F2, fam[k].gamma, fam[k].rc = (F1.data_ptr(), F2.data_ptr(),
                                                         g.data_ptr(), rc.data_ptr())
        fam[k].dims[:] = list(dims)
    prm = wb.bs._params(core, d, 1000.0, prec)
    pd = (C.c_longlong * 4)(*pshape)
    L.winds_bs_eval_device_noalloc.argtypes = [C.c_void_p, C.c_int, C.c_void_p,
                                               C.POINTER(C.c_longlong), C.c_void_p, C.c_void_p,
                                               C.c_void_p]
    return L.winds_bs_eval_device_noalloc(fam, len(dfams), dP.data_ptr(), pd, C.byref(prm),
                                          out.data_ptr(), C.c_void_p(stream))


def _compare(wb, dfams, dP, pshape, core, d, prec, stream):
    """One no-alloc call against winds_bs_eval_device on the same inputs."""
    import torch
    ref = torch.zeros(dP.numel(), dtype=torch.float64, device="cuda")
    out = torch.full_like(ref, float("nan"))  # every output element must be written
    wb.eval_device(dfams, (dP, pshape), core, d, 1000.0, ref, prec, stream=stream)
    wb.sync(stream)
    rc = _noalloc(wb, dfams, dP, pshape, out, core, d, stream, prec)
    assert rc == 0, wb.lib().winds_bs_last_error()
    u = out.cpu().numpy().reshape(pshape, order="F")
    u_ref = ref.cpu().numpy().reshape(pshape, order="F")
    assert np.all(np.isfinite(u))
    assert per_target_rel(u, u_ref) < (F32C_TOL if prec == "f32c" else F64_TOL)


def test_noalloc_matches_eval_device_on_two_calls(wb, synth):
    import torch
    torch.cuda.init()
    stream = torch.cuda.Stream()
    cases = [(synth.RotorCase(nst=21, nsteps=90, dpsi_deg=4.0, seed=12), wb.bs.CORE_VATISTAS, 2.0),
             (synth.RotorCase(nst=13, nsteps=40, dpsi_deg=6.0, seed=13), wb.bs.CORE_CUTOFF, 1e-4)]
    for prec in ("f32c", "f64"):
        for case, core, d in cases:  # two calls in a row, different sizes and core models
            dfams, dP, pshape = _device_inputs(wb, synth, case)
            _compare(wb, dfams, dP, pshape, core, d, prec, stream.cuda_stream)


def test_noalloc_at_its_target_limit_and_one_beyond(wb, synth):
    """Exactly WINDS_BS_NOALLOC_MAX_TARGETS targets (seeded points around a
    small wake) is evaluated like winds_bs_eval_device; one more is rejected."""
    import torch
    stream = torch.cuda.Stream()
    w = synth.make_wake(synth.RotorCase(nst=9, nsteps=24, dpsi_deg=10.0, seed=5))
    F1, F2 = synth.trail_filaments(w["dom"])
    dev = lambda a: torch.from_numpy(np.asarray(a).ravel(order="F").copy()).cuda()
    dfams = [(dev(F1), dev(F2), dev(w["gamma_trail"]), dev(w["rc_trail"]), F1.shape)]
    rng = np.random.default_rng(7)
    pts = rng.uniform(-70.0, 70.0, size=(MAX_TARGETS, 3))
    pts[:, 0] = rng.uniform(-5.0, 40.0, size=MAX_TARGETS)
    P = np.asfortranarray(pts.reshape(MAX_TARGETS, 3, 1, 1))
    _compare(wb, dfams, dev(P), P.shape, wb.bs.CORE_VATISTAS, 2.0, "f32c", stream.cuda_stream)
    over = np.asfortranarray(np.zeros((MAX_TARGETS + 1, 3, 1, 1)))
    out = torch.zeros(over.size, dtype=torch.float64, device="cuda")
    rc = _noalloc(wb, dfams, dev(over), over.shape, out, wb.bs.CORE_VATISTAS, 2.0, stream.cuda_stream)
    assert rc == 1  # WINDS_BS_ERR_ARG
    assert b"limited to" in wb.lib().winds_bs_last_error()


def test_noalloc_leaves_free_memory_unchanged(wb, synth):
    """After a first call, a second one changes the device's free memory by
    nothing: the call allocates no device memory."""
    import torch
    stream = torch.cuda.Stream()
    dfams, dP, pshape = _device_inputs(wb, synth, synth.RotorCase(nst=17, nsteps=60, seed=21))
    out = torch.zeros(dP.numel(), dtype=torch.float64, device="cuda")
    for prec in ("f32c", "f64"):
        assert _noalloc(wb, dfams, dP, pshape, out, wb.bs.CORE_VATISTAS, 2.0, stream.cuda_stream,
                        prec) == 0
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for prec in ("f32c", "f64"):
        assert _noalloc(wb, dfams, dP, pshape, out, wb.bs.CORE_VATISTAS, 2.0, stream.cuda_stream,
                        prec) == 0
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0


def test_noalloc_rejects_sizes_beyond_its_limit(wb, synth):
    import torch
    n = 131072 + 1  # WINDS_BS_NOALLOC_MAX_FILAMENTS + 1, one [n,3,1,1] family
    F = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
    g = torch.zeros(n, dtype=torch.float64, device="cuda")
    dP = torch.zeros(3, dtype=torch.float64, device="cuda")
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    rc = _noalloc(wb, [(F, F, g, g, (n, 3, 1, 1))], dP, (1, 3, 1, 1), out, wb.bs.CORE_CUTOFF, 1e-4, 0)
    assert rc == 1  # WINDS_BS_ERR_ARG
    assert b"limited to" in wb.lib().winds_bs_last_error()
