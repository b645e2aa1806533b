"""Writes tests/golden/nrel5mw.npz: the NREL 5-MW blade (trailing-node radius,
chord, aerodynamic twist, airfoil index) and its eight airfoil tables as the
reference's modeldata/NRELrotor.m and modeldata/NREL_files/*.dat give them,
plus the turbine constants of NRELrotor.m:60-72 and the overhang default of
WInDS.m:64. Run where the reference tree is available:

    python tests/golden/make_nrel.py /path/to/WInDS-Master

Only numbers are taken from NRELrotor.m: each vector token must be a number,
a quotient of two numbers, or blade.HubRad / blade.TipRad.
"""
from __future__ import annotations

import importlib
import os
import re
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
NUM = r"[-+]?\d*\.?\d+(?:[eE][-+]?\d+)?"


def _vector(src: str, name: str, names: dict) -> np.ndarray:
    m = re.search(rf"{re.escape(name)}\s*=\s*(-?)\[(.*?)\]", src, re.S)
    if not m:
        raise ValueError(f"{name} not found")
    sign = -1.0 if m.group(1) == "-" else 1.0
    body = m.group(2).replace("...", " ")
    out = []
    for tok in body.split():
        if tok in names:
            out.append(names[tok])
        elif re.fullmatch(NUM, tok):
            out.append(float(tok))
        elif re.fullmatch(rf"{NUM}/{NUM}", tok):
            a, b = tok.split("/")
            out.append(float(a) / float(b))
        else:
            raise ValueError(f"unexpected token {tok!r} in {name}")
    return sign * np.asarray(out)


def _scalar(src: str, name: str) -> float:
    m = re.search(rf"{re.escape(name)}\s*=\s*({NUM})\s*;", src)
    if not m:
        raise ValueError(f"{name} not found")
    return float(m.group(1))


def main(ref: str) -> None:
    sys.path.insert(0, ROOT)
    md = importlib.import_module("winds-master_b200.modeldata")
    src = open(os.path.join(ref, "modeldata", "NRELrotor.m")).read()
    names = {"blade.HubRad": _scalar(src, "blade.HubRad"), "blade.TipRad": _scalar(src, "blade.TipRad")}
    r = _vector(src, "blade.RTrail", names)
    chord = _vector(src, "blade.ChordTrail", names)
    twist = _vector(src, "blade.AeroTwstTrail", names)
    nfoil = _vector(src, "blade.NFoil", names).astype(np.int64)
    foils = re.search(r"airfoils\.Names\s*=\s*\{(.*?)\}", src, re.S).group(1)
    foil_names = re.findall(r"'([A-Za-z0-9_]+)'", foils)
    out = dict(r_trail=r, chord_trail=chord, twist_trail=twist, nfoil_trail=nfoil,
               names=np.array(foil_names), nb=3, tower_ht=_scalar(src, "turbine.TowerHt"),
               twr2shft=_scalar(src, "turbine.Twr2Shft"), shaft_tilt=_scalar(src, "turbine.ShftTilt"),
               precone=-2.5, overhang=5.0)
    for k, n in enumerate(foil_names):
        t = md.read_airfoil(os.path.join(ref, "modeldata", "NREL_files", n + ".dat"))
        for f in ("aoa", "cl", "cd"):
            out[f"{f}_{k}"] = t[f]
    np.savez_compressed(os.path.join(ROOT, "tests", "golden", "nrel5mw.npz"), **out)
    print("wrote nrel5mw.npz:", len(r), "trailing nodes,", len(foil_names), "airfoils")


if __name__ == "__main__":
    src_tree = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("WINDS_REFERENCE")
    if not src_tree:
        sys.exit("usage: make_nrel.py <reference tree>  (or set WINDS_REFERENCE)")
    main(src_tree)
