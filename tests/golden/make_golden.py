"""Generates the golden fixtures under tests/golden/ (run where the reference
tree and its compiled MEX exist: ``make -C oracle && python tests/golden/make_golden.py``).

Every fixture stores its inputs in WInDS layout and the outputs of
  * ``u_oracle``: the NumPy restatement of core/BiotSavart.m (oracle/biot_savart_ref.py),
  * ``u_ref``   : the reference's own compiled MEX host loop (cut-off cases only;
                  cuda/source/BiotSavartMex.cu:268-282 via oracle/_ref),
so the oracle is pinned against the reference and the GPU paths against both.
"""
from __future__ import annotations

import importlib
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import biot_savart_ref as ref  # noqa: E402
import oracle as orc  # noqa: E402

synth = importlib.import_module("winds-master_b200.synth")


def small_case():
    return synth.RotorCase(nst=5, nsteps=6, dpsi_deg=10.0, seed=11)


def wake_fixture(name, d, with_ref):
    w = synth.make_wake(small_case())
    out = {}
    for fam, (F1, F2), g, rc in (("shed", synth.shed_filaments(w["dom"]), w["gamma_shed"], w["rc_shed"]),
                                 ("trail", synth.trail_filaments(w["dom"]), w["gamma_trail"], w["rc_trail"])):
        for tname, P in (("wake", w["dom"]), ("ll", w["ll"])):
            u, _ = ref.biot_savart(F1, F2, P, g, rc, d, 1000.0, "full")
            key = f"{fam}_{tname}"
            out[f"u_oracle_{key}"] = u
            if with_ref:
                out[f"u_ref_{key}"] = orc.ref_host_eval(F1, F2, P, g, rc, d, 1000.0)
        out[f"F1_{fam}"], out[f"F2_{fam}"], out[f"g_{fam}"], out[f"rc_{fam}"] = F1, F2, g, rc
    out["P_wake"], out["P_ll"] = w["dom"], w["ll"]
    out["d"] = np.array(str(d))
    np.savez_compressed(os.path.join(HERE, name), **out)


def edge_fixture():
    """Edge cases of core/BiotSavart.m:111 and degenerate geometry."""
    rng = np.random.Generator(np.random.PCG64(3))
    x1 = rng.uniform(-2, 2, size=(6, 3))
    x2 = x1 + rng.uniform(-1, 1, size=(6, 3))
    x2[1] = x1[1]                      # zero-length filament
    g = rng.uniform(-3, 3, size=6)
    g[2] = np.nan                      # NaN circulation: term zeroed
    g[3] = 0.0
    rc = rng.uniform(0.01, 0.2, size=6)
    pts = rng.uniform(-3, 3, size=(9, 3))
    pts[0] = x1[0]                     # target on an endpoint
    pts[1] = 0.5 * (x1[4] + x2[4])     # target on a filament
    pts[2] = x1[5] + 3.0 * (x2[5] - x1[5])  # target on a filament's extension
    pts[3] = np.array([40.0, 0.0, 0.0])     # beyond co for every filament
    F1 = np.asfortranarray(x1.reshape(6, 3, 1, 1))
    F2 = np.asfortranarray(x2.reshape(6, 3, 1, 1))
    P = np.asfortranarray(pts.reshape(9, 3, 1, 1))
    G = np.asfortranarray(g.reshape(6, 1, 1, 1))
    R = np.asfortranarray(rc.reshape(6, 1, 1, 1))
    out = dict(F1=F1, F2=F2, P=P, g=G, rc=R)
    for d in (1e-4, "visc2"):
        for co in (1000.0, 5.0):
            u, _ = ref.biot_savart(F1, F2, P, G, R, d, co, "full")
            out[f"u_oracle_{d}_{co}"] = u
    np.savez_compressed(os.path.join(HERE, "bs_edge.npz"), **out)


def kat_fixture():
    """Analytic known answers: straight segment and regular N-gon ring centre."""
    out = {}
    # straight segment from (0,0,-a) to (0,0,b), point at (h,0,0): inviscid
    # |u| = G/(4 pi h) (cos t1 + cos t2), direction +y for G > 0 along +z.
    a, b, h, G = 1.3, 2.1, 0.7, 2.5
    out["seg_u"] = np.array([0.0, G / (4 * math.pi * h) * (a / math.hypot(a, h) + b / math.hypot(b, h)), 0.0])
    out["seg_geom"] = np.array([a, b, h, G])
    # N-gon of circumradius R in the y-z plane, circulation G: |u| at the centre
    # = N G tan(pi/N) / (2 pi R) along the axis.
    N, R = 64, 3.0
    out["ring_u"] = np.array([N * G * math.tan(math.pi / N) / (2 * math.pi * R)])
    out["ring_geom"] = np.array([N, R, G])
    np.savez_compressed(os.path.join(HERE, "bs_kat.npz"), **out)


if __name__ == "__main__":
    with_ref = orc.ref_available()
    if not with_ref:
        print("reference MEX not built: cut-off fixtures carry no u_ref")
    wake_fixture("bs_small_cutoff.npz", 1e-4, with_ref)
    wake_fixture("bs_small_visc2.npz", "visc2", False)
    edge_fixture()
    kat_fixture()
    print("written to", HERE)
