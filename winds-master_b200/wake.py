"""ctypes binding of ``include/winds_wake.h``: the device-resident free-wake
time step of many rotor cases at once (the WInDS main loop's induced
velocity, bookkeeping, core growth and convection: ``WInDS.m:127-179``).

``WakeBatch(cases, ...)`` takes case dicts as :func:`synth.make_wake_case`
returns them (WInDS-layout arrays), ``step(n, graph=True)`` advances every
case, ``state(i)`` reads one case back.

A case dict may also give ``na_start`` (live age columns at step 0: 2 starts
from the two columns of ``core/initials.m:84-86`` and grows one column per
step up to ``na``), ``time`` (``fastout.Time`` per step) and ``r0_step``
(``wake.r0`` per step, ``core/initials.m:134-135``). ``startup="reference"``
applies the reference's time-index switches (``ab2.m:35``, ``ab4.m:35``,
``pcc.m:40``, ``filamentmod.m:26``; no lifting-line iteration at step 0).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .bs import _check, lib, parse_core

INTEG = {"fe": 0, "ab2": 1, "ab4": 2, "pcc": 3}


class WakeCaseC(C.Structure):
    _fields_ = [("nst", C.c_int), ("nb", C.c_int), ("na", C.c_int), ("nsteps", C.c_int),
                ("dt", C.c_double), ("t0", C.c_double),
                ("quarter", C.c_void_p), ("trailing", C.c_void_p), ("wind", C.c_void_p),
                ("shear", C.c_double), ("hub_height", C.c_double), ("core_mode", C.c_int),
                ("r0", C.c_double), ("rc0", C.c_double), ("alpha", C.c_double), ("nu", C.c_double),
                ("a1", C.c_double), ("delta", C.c_double),
                ("dom", C.c_void_p), ("bound", C.c_void_p), ("trail_gamma", C.c_void_p),
                ("na_start", C.c_int), ("time", C.c_void_p), ("r0_step", C.c_void_p)]


class KJCaseC(C.Structure):
    _fields_ = [("ll", C.c_void_p), ("bxn", C.c_void_p), ("byn", C.c_void_p), ("bzn", C.c_void_p),
                ("vblade", C.c_void_p), ("chord", C.c_void_p), ("foil", C.c_void_p),
                ("n_foils", C.c_int), ("foil_points", C.c_void_p), ("aoa", C.c_void_p),
                ("cl", C.c_void_p), ("cd", C.c_void_p), ("r_over_R", C.c_void_p),
                ("chord_over_R", C.c_void_p), ("twist", C.c_void_p), ("azimuth", C.c_void_p),
                ("r_station", C.c_void_p), ("dr_station", C.c_void_p), ("rpm", C.c_void_p),
                ("rho", C.c_double), ("pitch", C.c_void_p)]


class KJParamsC(C.Structure):
    _fields_ = [("relax", C.c_double), ("tol", C.c_double), ("maxiter", C.c_int),
                ("ll_fp64", C.c_int)]


class WakeParamsC(C.Structure):
    _fields_ = [("integrator", C.c_int), ("core_model", C.c_int), ("d", C.c_double),
                ("co", C.c_double), ("precision", C.c_int), ("pcc_double_add", C.c_int),
                ("stretch", C.c_int), ("startup", C.c_int)]

STARTUP = {"full": 0, "reference": 1}


def _bind():
    L = lib()
    if not hasattr(L, "_wake_bound"):
        L.winds_wake_create.argtypes = [C.POINTER(WakeCaseC), C.c_int, C.POINTER(WakeParamsC),
                                        C.POINTER(C.c_void_p)]
        L.winds_wake_step.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.winds_wake_get_state.argtypes = [C.c_void_p, C.c_int] + [C.c_void_p] * 7
        L.winds_wake_set_bound.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.winds_wake_stats.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_longlong),
                                       C.POINTER(C.c_int)]
        L.winds_wake_destroy.argtypes = [C.c_void_p]
        L.winds_wake_set_kj.argtypes = [C.c_void_p, C.POINTER(KJCaseC), C.POINTER(KJParamsC)]
        L.winds_wake_kj_stats.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_longlong)]
        L.winds_wake_get_perf.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        L.winds_wake_set_mlp.argtypes = [C.c_void_p, C.c_void_p]
        L.winds_wake_get_kj_guess.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.winds_wake_get_kj_features.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.winds_wake_get_loads.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.winds_wake_get_live.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int),
                                          C.POINTER(C.c_longlong)]
        L._wake_bound = True
    return L


class WakeBatch:
    def __init__(self, cases, integrator="pcc", d="visc2", co=1000.0, precision="f32c",
                 pcc_double_add=True, stretch=True, startup="full"):
        L = _bind()
        self._keep = []
        arr = (WakeCaseC * len(cases))()
        for k, c in enumerate(cases):
            a = arr[k]
            for f in ("nst", "nb", "na", "nsteps", "core_mode"):
                setattr(a, f, int(c[f]))
            for f in ("dt", "t0", "shear", "hub_height", "r0", "rc0", "alpha", "nu", "a1", "delta"):
                setattr(a, f, float(c[f]))
            for f in ("quarter", "trailing", "wind", "dom", "bound", "trail_gamma"):
                x = np.asfortranarray(c[f], dtype=np.float64)
                self._keep.append(x)
                setattr(a, f, x.ctypes.data)
            a.na_start = int(c.get("na_start", 0))
            for f in ("time", "r0_step"):
                if c.get(f) is not None:
                    x = np.ascontiguousarray(c[f], dtype=np.float64)
                    if x.size < int(c["nsteps"]):
                        raise ValueError(f"case {k}: {f} has {x.size} entries, nsteps is {c['nsteps']}")
                    self._keep.append(x)
                    setattr(a, f, x.ctypes.data)
        core, dv = parse_core(d)
        p = WakeParamsC(INTEG[integrator], core, dv, float(co),
                        {"f32c": 0, "f64": 1}[precision], int(pcc_double_add), int(stretch),
                        STARTUP[startup])
        h = C.c_void_p()
        _check(L.winds_wake_create(arr, len(cases), C.byref(p), C.byref(h)))
        self.h = h
        self.cases = [dict(nst=c["nst"], nb=c["nb"], na=c["na"]) for c in cases]

    def step(self, n=1, graph=False):
        _check(_bind().winds_wake_step(self.h, int(n), 1 if graph else 0))

    def live(self, i=0):
        """(live age columns of case ``i``'s wake now, steps run so far)."""
        m, st = C.c_int(), C.c_longlong()
        _check(_bind().winds_wake_get_live(self.h, i, C.byref(m), C.byref(st)))
        return m.value, st.value

    def state(self, i):
        c = self.cases[i]
        nst, nb, na = c["nst"], c["nb"], c["na"]
        ns = nst - 1
        out = dict(dom=np.zeros((nst, 3, na, nb), order="F"), bound=np.zeros((ns, nb), order="F"),
                   shed=np.zeros((ns, na, nb), order="F"), trail=np.zeros((nst, na - 1, nb), order="F"),
                   rc_shed=np.zeros((ns, na, nb), order="F"),
                   rc_trail=np.zeros((nst, na - 1, nb), order="F"),
                   uind=np.zeros((nst, 3, na, nb), order="F"))
        ks = ("dom", "bound", "shed", "trail", "rc_shed", "rc_trail", "uind")
        _check(_bind().winds_wake_get_state(self.h, i, *[out[k].ctypes.data for k in ks]))
        return out

    def bound(self, i):
        """Bound circulation [ns, nb] of case ``i``."""
        c = self.cases[i]
        g = np.zeros((c["nst"] - 1, c["nb"]), order="F")
        _check(_bind().winds_wake_get_state(self.h, i, None, g.ctypes.data, None, None, None, None,
                                            None))
        return g

    def set_bound(self, i, bound):
        b = np.asfortranarray(bound, dtype=np.float64)
        _check(_bind().winds_wake_set_bound(self.h, i, b.ctypes.data))

    def set_kj(self, kjs, relax=0.25, tol=1e-6, maxiter=30, ll_fp64=False):
        """Attaches one lifting line per case (dicts as :func:`synth.make_kj_case`
        returns them): every later step runs the Kutta-Joukowski iteration
        (``ll_fp64``: its lifting-line evaluations in FP64 in an FP32c batch)."""
        arr = (KJCaseC * len(kjs))()
        for k, j in enumerate(kjs):
            a = arr[k]
            for f in ("ll", "bxn", "byn", "bzn", "vblade", "chord", "aoa", "cl", "cd"):
                x = np.asfortranarray(j[f], dtype=np.float64)
                self._keep.append(x)
                setattr(a, f, x.ctypes.data)
            for f in ("foil", "foil_points"):
                x = np.ascontiguousarray(j[f], dtype=np.int32)
                self._keep.append(x)
                setattr(a, f, x.ctypes.data)
            a.n_foils = len(j["foil_points"])
            # MLP and loads inputs, optional
            for f in ("r_over_R", "chord_over_R", "twist", "azimuth", "r_station", "dr_station", "rpm",
                      "pitch"):
                if f in j:
                    x = np.asfortranarray(j[f], dtype=np.float64)
                    self._keep.append(x)
                    setattr(a, f, x.ctypes.data)
            a.rho = float(j.get("rho", 0.0))
        p = KJParamsC(float(relax), float(tol), int(maxiter), int(bool(ll_fp64)))
        _check(_bind().winds_wake_set_kj(self.h, arr, C.byref(p)))

    def set_mlp(self, mlp):
        """Start every later step's iteration from ``mlp``'s prediction
        (``None``: from the previous step's bound circulation)."""
        _check(_bind().winds_wake_set_mlp(self.h, mlp.h if mlp is not None else None))
        self._mlp = mlp  # the network must outlive its use

    def kj_guess(self, i):
        """Start value [ns, nb] of case ``i``'s last iteration."""
        c = self.cases[i]
        g = np.zeros((c["nst"] - 1, c["nb"]), order="F")
        _check(_bind().winds_wake_get_kj_guess(self.h, i, g.ctypes.data))
        return g

    def loads(self):
        """Rotor thrust (N), torque (N m), power (W) of every case at the last
        step (postproc/perform.m)."""
        n = len(self.cases)
        T, Q, P = np.zeros(n), np.zeros(n), np.zeros(n)
        _check(_bind().winds_wake_get_loads(self.h, T.ctypes.data, Q.ctypes.data, P.ctypes.data))
        return T, Q, P

    def kj_features(self, i):
        """MLP features [ns*nb, 11] of case ``i`` at the last step."""
        c = self.cases[i]
        x = np.zeros(((c["nst"] - 1) * c["nb"], 11), dtype=np.float32)
        _check(_bind().winds_wake_get_kj_features(self.h, i, x.ctypes.data))
        return x

    def kj_stats(self):
        """(iterations [ncases], residual [ncases], lifting-line evaluations)
        of the last step."""
        n = len(self.cases)
        it = np.zeros(n, dtype=np.int32)
        res = np.zeros(n)
        ev = C.c_longlong()
        _check(_bind().winds_wake_kj_stats(self.h, it.ctypes.data, res.ctypes.data, C.byref(ev)))
        return it, res, ev.value

    def perf(self, i):
        """Cl, Cd, AoA [ns, nb] of case ``i`` from the last iteration."""
        c = self.cases[i]
        shp = (c["nst"] - 1, c["nb"])
        cl, cd, aoa = (np.zeros(shp, order="F") for _ in range(3))
        _check(_bind().winds_wake_get_perf(self.h, i, cl.ctypes.data, cd.ctypes.data, aoa.ctypes.data))
        return cl, cd, aoa

    def stats(self):
        ms, n, l = C.c_double(), C.c_longlong(), C.c_int()
        _check(_bind().winds_wake_stats(self.h, C.byref(ms), C.byref(n), C.byref(l)))
        return ms.value, n.value, l.value

    def close(self):
        if getattr(self, "h", None):
            _bind().winds_wake_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
