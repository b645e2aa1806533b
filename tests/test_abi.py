"""CPU tests of the drop-in boundary: the library loads, exports every symbol
include/*.h declares, and its mexFunction keeps the reference's argument
contract and error behaviour (cuda/source/BiotSavartMex.cu:688-807). No
compute call reaches a GPU here."""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT


def declared_functions():
    names = set()
    for h in ("winds_bs.h", "mex.h", "matrix.h", "winds_wake.h", "winds_mlp.h", "winds_kin.h"):
        path = os.path.join(ROOT, "include", h)
        if not os.path.exists(path):
            continue
        text = open(path).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", text):
            name = m.group(1)
            if name.startswith(("winds_", "mx", "mex")) and not name.startswith(("mxArray", "mex_function")):
                names.add(name)
    return sorted(names)


def test_library_exports_every_declared_symbol(wb):
    lib = C.CDLL(wb.LIB_PATH)
    names = declared_functions()
    assert "winds_bs_eval_device" in names and "mexFunction" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def _args(synth, **over):
    w = synth.make_wake(synth.RotorCase(nst=5, nsteps=4))
    F1, F2 = synth.shed_filaments(w["dom"])
    a = dict(F1=F1, F2=F2, P=w["dom"], gamma=w["gamma_shed"], rc=w["rc_shed"], d=1e-4,
             cmod="none", co=1000.0, type_="fuln", gpu="true", gpuhw=np.array([128.0, 1.0, 0.0]))
    a.update(over)
    return a


def _call(wb, nlhs, a, drop_last=False):
    mexcall = __import__("importlib").import_module("winds-master_b200.mexcall")
    lib = mexcall.MexLib(wb.LIB_PATH)
    vals = [a["F1"], a["F2"], a["P"], a["gamma"], a["rc"], a["d"], a["cmod"], a["co"], a["type_"],
            a["gpu"], a["gpuhw"]]
    if drop_last:
        vals = vals[:-1]
    return lib.call(nlhs, *vals)


def test_mex_requires_11_inputs(wb, synth, oracle):
    mexcall = __import__("importlib").import_module("winds-master_b200.mexcall")
    with pytest.raises(mexcall.MexError, match="11 inputs expected"):
        _call(wb, 2, _args(synth), drop_last=True)
    if oracle.ref_available():  # same message from the reference's own MEX
        a = _args(synth)
        with pytest.raises(mexcall.MexError, match="11 inputs expected"):
            oracle.ref_mex().call(2, a["F1"], a["F2"], a["P"], a["gamma"], a["rc"], a["d"], a["cmod"],
                                  a["co"], a["type_"], a["gpu"])


def test_mex_requires_2_outputs(wb, synth):
    mexcall = __import__("importlib").import_module("winds-master_b200.mexcall")
    with pytest.raises(mexcall.MexError, match="2 outputs expected"):
        _call(wb, 1, _args(synth))


@pytest.mark.parametrize("over,ident", [
    (dict(cmod="bogus"), "winds:bs:cmod"),
    (dict(gamma=np.zeros((3, 1))), "winds:bs:gdims"),
    (dict(P=np.zeros((2, 3, 1, 1, 2))), "winds:bs:pdims"),
    (dict(P=np.zeros((4, 2, 1, 1))), "winds:bs:pdims"),
    (dict(cmod=1.0), "winds:bs:type"),
])
def test_mex_argument_errors(wb, synth, over, ident):
    mexcall = __import__("importlib").import_module("winds-master_b200.mexcall")
    with pytest.raises(mexcall.MexError) as ei:
        _call(wb, 2, _args(synth, **over))
    assert ei.value.identifier == ident


def test_mex_output_shapes_and_leng(wb, synth, ref):
    """'leng' needs no device: L(i) = |F2-F1| for i < min(#P,#F); uind zeros
    shaped like P, L shaped [P1,1,P3,P4] (BiotSavartMex.cu:776-783)."""
    a = _args(synth, type_="leng", gpuhw=np.array([128.0, 1.0]))
    uind, L = _call(wb, 2, a)
    assert uind.shape == a["P"].shape and not uind.any()
    assert L.shape == (a["P"].shape[0], 1) + a["P"].shape[2:]
    lens = ref.filament_length(a["F1"], a["F2"]).ravel(order="F")
    n = min(lens.size, L.size)
    np.testing.assert_allclose(L.ravel(order="F")[:n], lens[:n], rtol=1e-15)


def test_mex_unknown_type_returns_zeros(wb, synth):
    a = _args(synth, type_="none", gpuhw=np.array([128.0]))
    uind, L = _call(wb, 2, a)
    assert not uind.any() and not L.any()


def test_no_cpu_fallback(wb, synth):
    """Without a GPU the engine fails loudly instead of computing on the CPU."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    mexcall = __import__("importlib").import_module("winds-master_b200.mexcall")
    with pytest.raises(mexcall.MexError, match="no CUDA device"):
        _call(wb, 2, _args(synth))
    a = _args(synth)
    with pytest.raises(wb.WindsError) as ei:
        wb.BiotSavart(a["F1"], a["F2"], a["P"], a["gamma"], a["rc"], 1e-4, 1000.0, "full")
    assert ei.value.code == 5


def test_biotsavart_length_and_nonfull_types(wb, synth, ref):
    """BiotSavart(...,'length') and unknown types need no device and follow
    core/BiotSavart.m:74-77."""
    a = _args(synth)
    u, L = wb.BiotSavart(a["F1"], a["F2"], a["P"], a["gamma"], a["rc"], 1e-4, 1000.0, "length")
    u_r, L_r = ref.biot_savart(a["F1"], a["F2"], a["P"], a["gamma"], a["rc"], 1e-4, 1000.0, "length")
    np.testing.assert_array_equal(L, L_r)
    assert u.shape == u_r.shape and not u.any()
