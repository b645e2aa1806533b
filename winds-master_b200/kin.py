"""ctypes binding of ``include/winds_kin.h``: blade positions, frames and
blade-frame velocities of ``core/kinematics.m`` and ``core/velocity.m``,
evaluated on the GPU.

``kinematics(r)`` takes a dict with the turbine time series and geometry
(``time, azimuth, pitch [nt, nb], nac_yaw, ptfm [nt, 6], wind [nt, 3],
r_trail, chord_trail, twist_trail, r_nodes, chord, twist, precone [nb],
overhang, shaft_tilt, tower_ht, twr2shft, ptfm_ref``; angles in degrees) and
returns the WInDS-layout arrays (``hub [nt, 3]``; ``lead, quarter, trail,
bxt, byt, bzt [nst, 3, nt, nb]``; ``bound, colloc, end, bxn, byn, bzn,
vbound, vblade [ns, 3, nt, nb]``).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .bs import _check, lib

_IN = ("time", "azimuth", "pitch", "nac_yaw", "ptfm", "wind", "r_trail", "chord_trail", "twist_trail",
       "r_nodes", "chord", "twist", "precone")
_SCALARS = ("overhang", "shaft_tilt", "tower_ht", "twr2shft")
_OUT_T = ("lead", "quarter", "trail")
_OUT_S = ("bound", "colloc", "end")
_OUT_FT = ("bxt", "byt", "bzt")
_OUT_FS = ("bxn", "byn", "bzn", "vbound", "vblade")


class KinRotorC(C.Structure):
    _fields_ = ([("nt", C.c_int), ("nb", C.c_int), ("nst", C.c_int), ("ns", C.c_int)]
                + [(f, C.c_void_p) for f in _IN[:-1]] + [("precone", C.c_void_p)]
                + [(f, C.c_double) for f in _SCALARS] + [("ptfm_ref", C.c_double)])


class KinOutC(C.Structure):
    _fields_ = [(f, C.c_void_p) for f in ("hub",) + _OUT_T + _OUT_S + _OUT_FT + _OUT_FS]


def _bind():
    L = lib()
    if not hasattr(L, "_kin_bound"):
        L.winds_kinematics.argtypes = [C.POINTER(KinRotorC), C.POINTER(KinOutC)]
        L._kin_bound = True
    return L


def kinematics(r: dict) -> dict:
    keep = {f: np.asfortranarray(r[f], dtype=np.float64) for f in _IN}
    nt, nb = keep["time"].size, keep["precone"].size
    nst, ns = keep["r_trail"].size, keep["r_nodes"].size
    a = KinRotorC(nt, nb, nst, ns)
    for f in _IN:
        setattr(a, f, keep[f].ctypes.data)
    for f in _SCALARS + ("ptfm_ref",):
        setattr(a, f, float(r[f]))
    out = {"hub": np.zeros((nt, 3), order="F")}
    for f in _OUT_T + _OUT_FT:
        out[f] = np.zeros((nst, 3, nt, nb), order="F")
    for f in _OUT_S + _OUT_FS:
        out[f] = np.zeros((ns, 3, nt, nb), order="F")
    o = KinOutC(*[out[f].ctypes.data for f in ("hub",) + _OUT_T + _OUT_S + _OUT_FT + _OUT_FS])
    _check(_bind().winds_kinematics(C.byref(a), C.byref(o)))
    return out
