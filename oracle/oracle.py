"""ctypes front end of the C oracle and of the compiled reference MEX
(test infrastructure; see biot_savart_ref.py for the NumPy restatement).

``c_eval``   -- oracle/bs_oracle.c (FP64 restatement of core/BiotSavart.m,
                OpenMP over targets).
``ref_mex``  -- oracle/_ref/libref_bsmex.so: the reference's own
                cuda/source/BiotSavartMex.cu built by oracle/Makefile; its
                host branch (gpu='false') runs BiotSavart_nogpu
                (BiotSavartMex.cu:268-282), the cut-off core only.
"""
from __future__ import annotations

import ctypes as C
import importlib
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
C_LIB = os.path.join(HERE, "libbs_oracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libref_bsmex.so")

_c = None


def build():
    """Builds the C oracle (and the reference MEX when the reference tree exists)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True, capture_output=True)


def c_lib():
    global _c
    if _c is None:
        if not os.path.exists(C_LIB):
            build()
        L = C.CDLL(C_LIB)
        L.bs_oracle_eval.argtypes = [C.c_void_p] * 4 + [C.POINTER(C.c_longlong), C.c_void_p,
                                     C.POINTER(C.c_longlong), C.c_int, C.c_double, C.c_double,
                                     C.c_void_p, C.c_int]
        L.bs_oracle_length.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_longlong), C.c_void_p]
        _c = L
    return _c


def _d4(shape):
    d = list(shape) + [1] * (4 - len(shape))
    return (C.c_longlong * 4)(*d), d


def c_eval(F1, F2, P, gamma, rc, d, co, nthreads=0):
    """FP64 ``BiotSavart(...,'full')`` via the C restatement; ``d`` numeric or 'viscN'."""
    L = c_lib()
    F1 = np.asfortranarray(F1, dtype=np.float64)
    F2 = np.asfortranarray(F2, dtype=np.float64)
    P = np.asfortranarray(P, dtype=np.float64)
    g = np.asfortranarray(gamma, dtype=np.float64)
    r = np.asfortranarray(rc, dtype=np.float64)
    fd, _ = _d4(F1.shape)
    pd, pl = _d4(P.shape)
    if isinstance(d, str):
        s = d[d.index("visc") + 4:]
        n = float(s) if s.strip() else float("nan")
        visc, dv = (1, n) if n != 0 else (0, 0.0)
    else:
        visc, dv = 0, float(d)
    out = np.zeros(pl, order="F")
    L.bs_oracle_eval(F1.ctypes.data, F2.ctypes.data, g.ctypes.data, r.ctypes.data, fd,
                     P.ctypes.data, pd, visc, dv, float(co), out.ctypes.data, int(nthreads))
    return out


def c_eval_flat(x1, x2, gamma, rc, pts, d, co, nthreads=0):
    """Flat filaments ``[nf,3]`` and targets ``[np,3]`` -> ``[np,3]``."""
    F1 = np.asfortranarray(x1.reshape(-1, 3, 1, 1))
    F2 = np.asfortranarray(x2.reshape(-1, 3, 1, 1))
    P = np.asfortranarray(pts.reshape(-1, 3, 1, 1))
    g = np.asfortranarray(gamma.reshape(-1, 1, 1, 1))
    r = np.asfortranarray(rc.reshape(-1, 1, 1, 1))
    return c_eval(F1, F2, P, g, r, d, co, nthreads)[:, :, 0, 0]


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


_ref = None


def ref_mex():
    """:class:`MexLib` over the compiled reference MEX (raises if not built)."""
    global _ref
    if _ref is None:
        mexcall = importlib.import_module("winds-master_b200.mexcall")
        _ref = mexcall.MexLib(REF_LIB)
    return _ref


def ref_host_eval(F1, F2, P, gamma, rc, d, co):
    """``BiotSavartMex(F1,F2,P,gamma,rc,d,'none',co,'fuln','false',[128 1 0])``:
    the reference's serial host loop (cut-off core)."""
    u, _ = ref_mex().call(2, F1, F2, P, gamma, rc, float(d), "none", float(co), "fuln", "false",
                          np.array([128.0, 1.0, 0.0]))
    return u
