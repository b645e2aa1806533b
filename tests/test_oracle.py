"""CPU tests of the oracle: pinned against the reference's compiled MEX host
loop, the golden fixtures and analytic known answers (no GPU needed)."""
from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import load_golden, per_target_rel


def test_golden_oracle_recomputes(ref):
    """The NumPy restatement reproduces its stored golden outputs exactly."""
    for name in ("bs_small_cutoff.npz", "bs_small_visc2.npz"):
        g = load_golden(name)
        d = str(g["d"])
        d = float(d) if "visc" not in d else d
        for fam in ("shed", "trail"):
            for tname in ("wake", "ll"):
                u, _ = ref.biot_savart(g[f"F1_{fam}"], g[f"F2_{fam}"], g[f"P_{tname}"], g[f"g_{fam}"],
                                       g[f"rc_{fam}"], d, 1000.0, "full")
                np.testing.assert_array_equal(u, g[f"u_oracle_{fam}_{tname}"])


def test_oracle_pinned_to_reference_mex():
    """Cut-off core: the oracle agrees with the reference's own compiled host
    loop (cuda/source/BiotSavartMex.cu:268-282) on the stored fixtures."""
    g = load_golden("bs_small_cutoff.npz")
    assert any(k.startswith("u_ref_") for k in g), "fixture lacks reference outputs"
    for fam in ("shed", "trail"):
        for tname in ("wake", "ll"):
            assert per_target_rel(g[f"u_oracle_{fam}_{tname}"], g[f"u_ref_{fam}_{tname}"]) < 1e-12


def test_reference_mex_reproduces_fixture(oracle):
    """When oracle/_ref is built, rerunning the reference MEX gives the stored
    bytes (the fixture was made from it)."""
    if not oracle.ref_available():
        pytest.skip("oracle/_ref not built")
    g = load_golden("bs_small_cutoff.npz")
    for fam in ("shed", "trail"):
        u = oracle.ref_host_eval(g[f"F1_{fam}"], g[f"F2_{fam}"], g["P_wake"], g[f"g_{fam}"],
                                 g[f"rc_{fam}"], 1e-4, 1000.0)
        np.testing.assert_array_equal(u, g[f"u_ref_{fam}_wake"])


@pytest.mark.parametrize("d", [1e-4, 0.0, "visc2"])
def test_c_oracle_matches_numpy(oracle, ref, synth, d):
    w = synth.make_wake(synth.RotorCase(nst=7, nsteps=9, seed=4))
    F1, F2 = synth.trail_filaments(w["dom"])
    u_np, _ = ref.biot_savart(F1, F2, w["dom"], w["gamma_trail"], w["rc_trail"], d, 1000.0, "full")
    u_c = oracle.c_eval(F1, F2, w["dom"], w["gamma_trail"], w["rc_trail"], d, 1000.0)
    assert per_target_rel(u_c, u_np) < 1e-12


def test_edge_fixture(ref):
    g = load_golden("bs_edge.npz")
    for d in (1e-4, "visc2"):
        for co in (1000.0, 5.0):
            u, _ = ref.biot_savart(g["F1"], g["F2"], g["P"], g["g"], g["rc"], d, co, "full")
            np.testing.assert_array_equal(u, g[f"u_oracle_{d}_{co}"])
    # beyond co for every filament: exactly zero (core/BiotSavart.m:111)
    assert np.all(g["u_oracle_0.0001_5.0"][3] == 0.0)
    # the NaN-circulation filament contributes nothing: outputs stay finite
    assert np.all(np.isfinite(g["u_oracle_visc2_1000.0"]))


def test_kat_straight_segment(ref):
    k = load_golden("bs_kat.npz")
    a, b, h, G = k["seg_geom"]
    F1 = np.array([0.0, 0.0, -a]).reshape(1, 3, 1, 1)
    F2 = np.array([0.0, 0.0, b]).reshape(1, 3, 1, 1)
    P = np.array([h, 0.0, 0.0]).reshape(1, 3, 1, 1)
    g = np.array([G]).reshape(1, 1, 1, 1)
    u, _ = ref.biot_savart(F1, F2, P, g, np.zeros((1, 1, 1, 1)), 0.0, 1e9, "full")
    np.testing.assert_allclose(u[0, :, 0, 0], k["seg_u"], rtol=1e-13, atol=1e-15)
    # Vatistas n=2: far outside the core it tends to the inviscid value, inside to 0
    far, _ = ref.biot_savart(F1, F2, P, g, np.full((1, 1, 1, 1), 1e-8), "visc2", 1e9, "full")
    np.testing.assert_allclose(far[0, :, 0, 0], k["seg_u"], rtol=1e-6, atol=1e-12)
    near, _ = ref.biot_savart(F1, F2, P, g, np.full((1, 1, 1, 1), 1e4), "visc2", 1e9, "full")
    assert np.linalg.norm(near[0, :, 0, 0]) < 1e-4 * np.linalg.norm(k["seg_u"])


def test_kat_ring_centre(ref):
    k = load_golden("bs_kat.npz")
    N, R, G = k["ring_geom"]
    N = int(N)
    th = 2 * math.pi * np.arange(N + 1) / N
    pts = np.stack([np.zeros(N + 1), R * np.cos(th), R * np.sin(th)], 1)
    F1 = pts[:-1].reshape(N, 3, 1, 1)
    F2 = pts[1:].reshape(N, 3, 1, 1)
    u, _ = ref.biot_savart(F1, F2, np.zeros((1, 3, 1, 1)), np.full((N, 1, 1, 1), G),
                           np.zeros((N, 1, 1, 1)), 0.0, 1e9, "full")
    np.testing.assert_allclose(abs(u[0, 0, 0, 0]), k["ring_u"][0], rtol=1e-13)
    assert abs(u[0, 1, 0, 0]) < 1e-12 and abs(u[0, 2, 0, 0]) < 1e-12


def test_bookkeeping_matches_synth(ref, synth):
    """WInDS.m:131-140 restated twice (oracle, generator) agree, and Kelvin's
    theorem holds: trailing columns sum to zero spanwise."""
    w = synth.make_wake(synth.RotorCase(nst=6, nsteps=5, seed=2))
    G = w["bound"]
    trail_prev = w["gamma_trail"][:, :, 1:, :]
    shed, trail = ref.bookkeeping(G[:, 0:1, :][:, None, :, :], trail_prev)
    np.testing.assert_allclose(trail, w["gamma_trail"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(shed, w["gamma_shed"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(trail.sum(axis=0), 0.0, atol=1e-12)


def test_length_type(ref, synth):
    w = synth.make_wake(synth.RotorCase(nst=5, nsteps=4))
    F1, F2 = synth.shed_filaments(w["dom"])
    _, L = ref.biot_savart(F1, F2, w["dom"], w["gamma_shed"], w["rc_shed"], 1e-4, 1000.0, "length")
    np.testing.assert_allclose(L, ref.filament_length(F1, F2), rtol=0, atol=0)
