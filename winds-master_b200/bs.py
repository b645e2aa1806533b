"""ctypes binding of ``include/winds_bs.h`` and the reference-shaped API.

Function names and argument meaning follow the reference:

* ``BiotSavart(F1, F2, P, gamma, rc, d, co, type)`` -- ``core/BiotSavart.m:1``.
  ``d`` is the squared cut-off (numeric) or ``'viscN'`` for the Vatistas core of
  index N (``:49-53``); ``type`` is ``'full'`` or ``'length'``; ``rc`` holds
  squared core radii. Returns ``(uind, L)``: ``uind`` shaped like ``P`` padded
  to 4-D and ``L = |F2-F1|^2`` (``'full'``) or ``|F2-F1|`` (``'length'``).
* ``BiotSavartMex(F1, F2, P, gamma, rc, d, cmod, co, type, gpu, gpuhw)`` --
  ``cuda/source/BiotSavartMex.cu:688-807``; goes through the library's
  ``mexFunction`` exactly as MATLAB would.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .mexcall import MexLib, MexError  # noqa: F401

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libwinds_bs.so")

WINDS_BS_OK = 0
ERR_NAMES = {1: "ARG", 2: "CUDA", 3: "TIMEOUT", 4: "NOMEM", 5: "NODEV", 6: "DIVERGED"}
CORE_CUTOFF, CORE_VATISTAS = 0, 1
PREC_F32C, PREC_F64 = 0, 1
FLAG_SEQUENTIAL = 1


class WindsError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"winds_bs error {code} ({ERR_NAMES.get(code, '?')}): {msg}")
        self.code = code


class Family(C.Structure):
    _fields_ = [("F1", C.c_void_p), ("F2", C.c_void_p), ("gamma", C.c_void_p), ("rc", C.c_void_p),
                ("dims", C.c_longlong * 4)]


class Params(C.Structure):
    _fields_ = [("core_model", C.c_int), ("d", C.c_double), ("co", C.c_double),
                ("precision", C.c_int), ("flags", C.c_int)]


_lib = None
_mex = None


def lib():
    """The loaded ``libwinds_bs.so``; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is not built: run winds-master_b200/build.py "
                               "(the engine has no CPU fallback)")
        L = C.CDLL(LIB_PATH, mode=os.RTLD_LOCAL | os.RTLD_NOW)
        L.winds_bs_version.restype = C.c_char_p
        L.winds_bs_last_error.restype = C.c_char_p
        L.winds_bs_eval_device.argtypes = [C.POINTER(Family), C.c_int, C.c_void_p,
                                           C.POINTER(C.c_longlong), C.POINTER(Params), C.c_void_p,
                                           C.c_void_p]
        L.winds_bs_eval_host.argtypes = [C.POINTER(Family), C.c_int, C.c_void_p,
                                         C.POINTER(C.c_longlong), C.POINTER(Params), C.c_void_p]
        L.winds_bs_length_device.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_longlong),
                                             C.c_void_p, C.c_void_p]
        L.winds_bs_last_stats.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_int),
                                          C.POINTER(C.c_longlong)]
        L.winds_bs_last_core_free.argtypes = [C.POINTER(C.c_longlong)]
        L.winds_bs_last_chained.argtypes = [C.POINTER(C.c_int)]
        L.winds_bs_sync.argtypes = [C.c_void_p]
        L.winds_bs_set_tuning.argtypes = [C.c_int, C.c_longlong, C.c_longlong, C.c_int, C.c_int,
                                          C.c_double]
        L.winds_bs_get_tuning.argtypes = [C.c_int, C.c_longlong, C.c_longlong,
                                          C.POINTER(C.c_int), C.POINTER(C.c_int),
                                          C.POINTER(C.c_double)]
        _lib = L
    return _lib


def _check(rc: int):
    if rc != WINDS_BS_OK:
        raise WindsError(rc, lib().winds_bs_last_error().decode())


def _dims4(shape):
    d = list(shape) + [1] * (4 - len(shape))
    if len(d) > 4:
        raise ValueError(f"arrays are at most 4-D (got {shape})")
    return d


def parse_core(d):
    """``(core_model, d)`` from BiotSavart.m's ``d`` argument (``:49-53``)."""
    if isinstance(d, str):
        if "visc" not in d:
            raise ValueError(f"d must be numeric or 'viscN' (got {d!r})")
        s = d[d.index("visc") + 4:]
        n = float(s) if s.strip() else float("nan")
        if n == 0:
            return CORE_CUTOFF, 0.0
        return CORE_VATISTAS, n
    return CORE_CUTOFF, float(d)


def _params(core, dval, co, precision, flags=0):
    p = Params()
    p.core_model = core
    p.d = dval
    p.co = float(co)
    p.precision = {"f32c": PREC_F32C, "f64": PREC_F64}[precision] if isinstance(precision, str) else int(precision)
    p.flags = flags
    return p


def eval_host(families, P, core, dval, co, precision="f32c", flags=0, out=None):
    """Induced velocity of host (NumPy) filament families at host points ``P``.

    ``families``: list of ``(F1, F2, gamma, rc)`` NumPy arrays in WInDS layout.
    Returns ``uind`` with ``P``'s (4-D padded) shape, Fortran order; ``out``,
    if given, is that array (float64, Fortran-contiguous, e.g. in pinned
    memory so the device-to-host copy needs no staging)."""
    L = lib()
    P = np.asfortranarray(P, dtype=np.float64)
    pd = _dims4(P.shape)
    keep = []
    fams = (Family * max(1, len(families)))()
    for k, (F1, F2, g, rc) in enumerate(families):
        F1 = np.asfortranarray(F1, dtype=np.float64)
        F2 = np.asfortranarray(F2, dtype=np.float64)
        g = np.asfortranarray(g, dtype=np.float64)
        rc = np.asfortranarray(rc, dtype=np.float64)
        keep += [F1, F2, g, rc]
        fams[k].F1, fams[k].F2 = F1.ctypes.data, F2.ctypes.data
        fams[k].gamma, fams[k].rc = g.ctypes.data, rc.ctypes.data
        fams[k].dims[:] = _dims4(F1.shape)
    if out is None:
        out = np.zeros(pd, order="F")
    elif (out.dtype != np.float64 or tuple(out.shape) != tuple(pd)
          or not out.flags.f_contiguous):
        raise ValueError(f"out must be a Fortran-contiguous float64 array of shape {tuple(pd)}")
    prm = _params(core, dval, co, precision, flags)
    _check(L.winds_bs_eval_host(fams, len(families), P.ctypes.data, (C.c_longlong * 4)(*pd),
                                C.byref(prm), out.ctypes.data))
    return out


def eval_device(families, P, core, dval, co, out, precision="f32c", stream=None, flags=0):
    """Device evaluation on torch CUDA tensors (float64, Fortran-contiguous data
    viewed as ``[n,3,m,k]``; pass ``tensor.data_ptr()``-compatible tensors).

    ``families``: list of ``(F1, F2, gamma, rc, dims)`` with device tensors and
    their WInDS dims; ``P``: ``(tensor, dims)``; ``out``: device tensor with
    room for ``3 * prod(P dims without the 3)`` doubles."""
    L = lib()
    fams = (Family * max(1, len(families)))()
    for k, (F1, F2, g, rc, dims) in enumerate(families):
        fams[k].F1, fams[k].F2 = F1.data_ptr(), F2.data_ptr()
        fams[k].gamma, fams[k].rc = g.data_ptr(), rc.data_ptr()
        fams[k].dims[:] = _dims4(dims)
    Pt, pdims = P
    prm = _params(core, dval, co, precision, flags)
    s = None if stream is None else C.c_void_p(stream)
    _check(L.winds_bs_eval_device(fams, len(families), Pt.data_ptr(),
                                  (C.c_longlong * 4)(*_dims4(pdims)), C.byref(prm), out.data_ptr(), s))


def sync(stream=None):
    _check(lib().winds_bs_sync(None if stream is None else C.c_void_p(stream)))


def last_stats():
    """``(main_kernel_ms, launches, near_pairs)`` of the last evaluation."""
    ms, n, near = C.c_double(), C.c_int(), C.c_longlong()
    _check(lib().winds_bs_last_stats(C.byref(ms), C.byref(n), C.byref(near)))
    return ms.value, n.value, near.value


def last_core_free():
    """Pairs of the last FP32c evaluation that took the core-free form
    (Vatistas: targets at least 54 core radii from the filament's line;
    cut-off: targets far enough that d |L|^2 is below FP32 resolution)."""
    n = C.c_longlong()
    _check(lib().winds_bs_last_core_free(C.byref(n)))
    return n.value


def last_chained():
    """True when the last FP32c evaluation ran on the chained filament stream
    (the autotuner's layout choice for its size bucket)."""
    n = C.c_int()
    _check(lib().winds_bs_last_chained(C.byref(n)))
    return bool(n.value)


def set_autotune(on: bool):
    _check(lib().winds_bs_set_autotune(1 if on else 0))


def set_tuning(core, n_targets, n_filaments, T, KF, waves=8.0):
    _check(lib().winds_bs_set_tuning(core, n_targets, n_filaments, T, KF, waves))


def set_layout(core, n_targets, n_filaments, chained):
    """Stream layout of a bucket's FP32c evaluations (chained or input order)."""
    L = lib()
    L.winds_bs_set_layout.argtypes = [C.c_int, C.c_longlong, C.c_longlong, C.c_int]
    _check(L.winds_bs_set_layout(core, n_targets, n_filaments, 1 if chained else 0))


def get_tuning(core, n_targets, n_filaments):
    T, KF, w = C.c_int(), C.c_int(), C.c_double()
    _check(lib().winds_bs_get_tuning(core, n_targets, n_filaments, C.byref(T), C.byref(KF), C.byref(w)))
    return T.value, KF.value, w.value


def BiotSavart(F1, F2, P, gamma, rc, d, co, type_="full", precision="f32c"):
    """``[uind, L] = BiotSavart(F1,F2,P,gamma,rc,d,co,type)`` (``core/BiotSavart.m:1``)
    evaluated by the GPU engine. ``type_``: ``'full'`` or ``'length'``."""
    F1 = np.asarray(F1, dtype=np.float64)
    F2 = np.asarray(F2, dtype=np.float64)
    fd = _dims4(F1.shape)
    F1 = F1.reshape(fd, order="F")
    F2 = F2.reshape(fd, order="F")
    D = F2 - F1
    Lsq = D[:, 0:1] ** 2 + D[:, 1:2] ** 2 + D[:, 2:3] ** 2
    if type_ == "length":
        return np.zeros(np.shape(P)), np.sqrt(Lsq)
    Pn = np.asarray(P, dtype=np.float64)
    pd = _dims4(Pn.shape)
    if type_ != "full":
        return np.zeros(pd, order="F"), Lsq
    core, dval = parse_core(d)
    g = np.asarray(gamma, dtype=np.float64).reshape((fd[0], 1, fd[2], fd[3]), order="F")
    r = np.asarray(rc, dtype=np.float64).reshape((fd[0], 1, fd[2], fd[3]), order="F")
    uind = eval_host([(F1, F2, g, r)], Pn.reshape(pd, order="F"), core, dval, co, precision)
    return uind, Lsq


def BiotSavartMex(F1, F2, P, gamma, rc, d, cmod, co, type_, gpu, gpuhw):
    """``[uind, L] = BiotSavartMex(...)`` through the library's ``mexFunction``."""
    global _mex
    lib()
    if _mex is None:
        _mex = MexLib(LIB_PATH)
    return _mex.call(2, F1, F2, P, gamma, rc, d, cmod, co, type_, gpu, gpuhw)
