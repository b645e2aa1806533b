"""GPU parity tests of the induced-velocity kernels against the oracle.

Tolerances (per-target relative error |du|/|u_ref| unless stated):
  * FP64 path vs oracle: 1e-12; bit-exact vs the reference's compiled host
    loop when run sequentially (cut-off core);
  * FP32-compensated path vs FP64 oracle: 1e-5.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import load_golden, per_target_rel

pytestmark = pytest.mark.gpu

F32C_TOL = 1e-5
F64_TOL = 1e-12


def _golden_cases():
    for name, d in (("bs_small_cutoff.npz", 1e-4), ("bs_small_visc2.npz", "visc2")):
        g = load_golden(name)
        for fam in ("shed", "trail"):
            for tname in ("wake", "ll"):
                yield name, d, fam, tname, g


def test_golden_f64_and_f32c(wb):
    for name, d, fam, tname, g in _golden_cases():
        core, dv = wb.bs.parse_core(d)
        fams = [(g[f"F1_{fam}"], g[f"F2_{fam}"], g[f"g_{fam}"], g[f"rc_{fam}"])]
        u64 = wb.eval_host(fams, g[f"P_{tname}"], core, dv, 1000.0, "f64")
        u32 = wb.eval_host(fams, g[f"P_{tname}"], core, dv, 1000.0, "f32c")
        uo = g[f"u_oracle_{fam}_{tname}"]
        assert per_target_rel(u64, uo) < F64_TOL, (name, fam, tname)
        assert per_target_rel(u32, uo) < F32C_TOL, (name, fam, tname)


def test_f64_sequential_bitexact_vs_reference_mex(wb):
    """Cut-off core, one pass per target in filament order: the same bits as
    the reference's serial host loop (cuda/source/BiotSavartMex.cu:268-282)."""
    g = load_golden("bs_small_cutoff.npz")
    for fam in ("shed", "trail"):
        for tname in ("wake", "ll"):
            fams = [(g[f"F1_{fam}"], g[f"F2_{fam}"], g[f"g_{fam}"], g[f"rc_{fam}"])]
            u = wb.eval_host(fams, g[f"P_{tname}"], wb.bs.CORE_CUTOFF, 1e-4, 1000.0, "f64",
                             flags=wb.bs.FLAG_SEQUENTIAL)
            np.testing.assert_array_equal(u, g[f"u_ref_{fam}_{tname}"])


def _wake_targets(w):
    return [w["dom"], w["ll"]]


def test_small_case_both_families_all_targets(wb, synth, oracle):
    """3 blades x 17 nodes x 60 steps at 10 deg: shed + trailing filaments in
    one launch onto all wake nodes and lifting-line points."""
    w = synth.make_wake(synth.RotorCase())
    fams = [synth.shed_filaments(w["dom"]) + (w["gamma_shed"], w["rc_shed"]),
            synth.trail_filaments(w["dom"]) + (w["gamma_trail"], w["rc_trail"])]
    for d in (1e-4, "visc2"):
        core, dv = wb.bs.parse_core(d)
        for P in _wake_targets(w):
            uo = sum(oracle.c_eval(F1, F2, P, g, rc, d, 1000.0) for F1, F2, g, rc in fams)
            u64 = wb.eval_host(fams, P, core, dv, 1000.0, "f64")
            u32 = wb.eval_host(fams, P, core, dv, 1000.0, "f32c")
            assert per_target_rel(u64, uo) < F64_TOL
            assert per_target_rel(u32, uo) < F32C_TOL


@pytest.fixture(scope="module")
def large(synth):
    """3 blades x 41 nodes x 720 steps at 1 deg: 175,080 filaments, 88,803 targets."""
    w = synth.make_wake(synth.large_case())
    x1, x2, g, rc = synth.flat_filaments(w)
    fams = [synth.shed_filaments(w["dom"]) + (w["gamma_shed"], w["rc_shed"]),
            synth.trail_filaments(w["dom"]) + (w["gamma_trail"], w["rc_trail"])]
    return w, fams, (x1, x2, g, rc)


def test_large_case_subset_vs_oracle(wb, synth, oracle, large):
    """4096 seeded targets (1% placed within 0.5 rc of a segment) against the
    FP64 oracle over all 175k filaments."""
    w, fams, (x1, x2, g, rc) = large
    rng = np.random.Generator(np.random.PCG64(7))
    allp = np.concatenate([synth.flat_points(w["dom"]), synth.flat_points(w["ll"])])
    n_near = 41
    pts = np.concatenate([allp[rng.choice(allp.shape[0], 4096 - n_near, replace=False)],
                          synth.near_singular_targets(x1, x2, rc, n_near, rng)])
    P = np.asfortranarray(pts.reshape(-1, 3, 1, 1))
    uo = oracle.c_eval_flat(x1, x2, g, rc, pts, "visc2", 1000.0)
    u32 = wb.eval_host(fams, P, wb.bs.CORE_VATISTAS, 2.0, 1000.0, "f32c")[:, :, 0, 0]
    err = np.linalg.norm(u32 - uo, axis=1) / np.linalg.norm(uo, axis=1)
    assert err.max() < F32C_TOL, err.max()
    assert err[-n_near:].max() < F32C_TOL


def test_large_case_full_f32c_vs_f64(wb, large):
    """All 88,803 targets: FP32-compensated against the FP64 GPU path (itself
    pinned to the oracle above), plus exact linearity in the circulation, on
    the input-order and the chained filament stream."""
    w, fams, _ = large
    P = w["dom"]
    nt = P.shape[0] * P.shape[2] * P.shape[3]
    nf = sum(f[0].shape[0] * f[0].shape[2] * f[0].shape[3] for f in fams)
    u64 = wb.eval_host(fams, P, wb.bs.CORE_VATISTAS, 2.0, 1000.0, "f64")
    fams2 = [(F1, F2, 2.0 * g, rc) for F1, F2, g, rc in fams]
    for chained in (False, True):
        wb.set_tuning(wb.bs.CORE_VATISTAS, nt, nf, 4, 64, 32.0)
        wb.set_layout(wb.bs.CORE_VATISTAS, nt, nf, chained)
        u32 = wb.eval_host(fams, P, wb.bs.CORE_VATISTAS, 2.0, 1000.0, "f32c")
        assert wb.last_chained() == chained
        assert per_target_rel(u32, u64) < F32C_TOL, chained
        u32x2 = wb.eval_host(fams2, P, wb.bs.CORE_VATISTAS, 2.0, 1000.0, "f32c")
        np.testing.assert_array_equal(u32x2, 2.0 * u32)


def test_every_tiling_agrees(wb, synth, oracle):
    """Each compiled (T, KF) tiling of the FP32 kernel gives the oracle's
    answer, on the input-order and the chained filament stream."""
    w = synth.make_wake(synth.RotorCase(nst=21, nsteps=90, dpsi_deg=4.0, seed=5))
    fams = [synth.shed_filaments(w["dom"]) + (w["gamma_shed"], w["rc_shed"]),
            synth.trail_filaments(w["dom"]) + (w["gamma_trail"], w["rc_trail"])]
    P = w["dom"]
    nt = P.shape[0] * P.shape[2] * P.shape[3]
    nf = sum(f[0].shape[0] * f[0].shape[2] * f[0].shape[3] for f in fams)
    uo = sum(oracle.c_eval(F1, F2, P, g, rc, "visc2", 1000.0) for F1, F2, g, rc in fams)
    uc = sum(oracle.c_eval(F1, F2, P, g, rc, 1e-4, 1000.0) for F1, F2, g, rc in fams)
    for T in (2, 3, 4, 8):
        for KF in (32, 64, 128):
            for waves in (1.0, 16.0):
                for chained in (False, True):
                    wb.set_tuning(wb.bs.CORE_VATISTAS, nt, nf, T, KF, waves)
                    wb.set_layout(wb.bs.CORE_VATISTAS, nt, nf, chained)
                    u = wb.eval_host(fams, P, wb.bs.CORE_VATISTAS, 2.0, 1000.0, "f32c")
                    assert wb.last_chained() == chained
                    assert per_target_rel(u, uo) < F32C_TOL, (T, KF, waves, chained)
                    wb.set_tuning(wb.bs.CORE_CUTOFF, nt, nf, T, KF, waves)
                    wb.set_layout(wb.bs.CORE_CUTOFF, nt, nf, chained)
                    u = wb.eval_host(fams, P, wb.bs.CORE_CUTOFF, 1e-4, 1000.0, "f32c")
                    assert per_target_rel(u, uc) < F32C_TOL, (T, KF, waves, chained)


def test_tiles_full_of_near_pairs(wb, oracle):
    """A compact ring of 64 short filaments with a 1 m core inside a cloud of
    1024 targets: every pair is near-singular, so each tile lists far more
    FP64 pairs than one pass of its list holds. All of them are counted and
    the sums match the FP64 oracle for every tiling and both stream layouts."""
    rng = np.random.default_rng(11)
    nf, nt = 64, 1024
    a = np.linspace(0.0, 2 * np.pi, nf + 1)
    ring = np.stack([np.cos(a), np.sin(a), 0.1 * np.sin(3 * a)], 1)
    F1 = np.asfortranarray(ring[:-1].reshape(nf, 3, 1, 1))
    F2 = np.asfortranarray(ring[1:].reshape(nf, 3, 1, 1))
    g = np.asfortranarray(rng.uniform(5.0, 15.0, (nf, 1, 1, 1)))
    rc = np.full((nf, 1, 1, 1), 1.0, order="F")
    P = np.asfortranarray(rng.uniform(-1.0, 1.0, (nt, 3, 1, 1)))
    fams = [(F1, F2, g, rc)]
    uo = oracle.c_eval(F1, F2, P, g, rc, "visc2", 1000.0)
    for T in (2, 4, 8):
        for KF in (32, 64):
            for chained in (False, True):
                wb.set_tuning(wb.bs.CORE_VATISTAS, nt, nf, T, KF, 4.0)
                wb.set_layout(wb.bs.CORE_VATISTAS, nt, nf, chained)
                u = wb.eval_host(fams, P, wb.bs.CORE_VATISTAS, 2.0, 1000.0, "f32c")
                assert wb.last_stats()[2] == nf * nt, (T, KF, chained)
                assert per_target_rel(u, uo) < 1e-6, (T, KF, chained)


def test_edge_cases_gpu(wb):
    """Zero-length filament, NaN circulation, targets on an endpoint, on a
    filament and on its extension, and the reach cut-off co."""
    g = load_golden("bs_edge.npz")
    fams = [(g["F1"], g["F2"], g["g"], g["rc"])]
    for d in (1e-4, "visc2"):
        core, dv = wb.bs.parse_core(d)
        for co in (1000.0, 5.0):
            uo = g[f"u_oracle_{d if isinstance(d, str) else '0.0001'}_{co}"]
            scale = np.abs(uo).max()
            for prec, tol in (("f64", F64_TOL), ("f32c", F32C_TOL)):
                u = wb.eval_host(fams, g["P"], core, dv, co, prec)
                assert np.all(np.isfinite(u))
                assert np.abs(u - uo).max() <= tol * scale, (d, co, prec)
            if co == 5.0:
                assert np.all(u[3] == 0.0)


def _count(shape):
    d = list(shape) + [1] * (4 - len(shape))
    return d[0] * d[2] * d[3]


def test_chained_stream_on_unlinked_and_edge_inputs(wb, synth, oracle):
    """The chained filament stream evaluates any input correctly, linked or
    not: the edge cases above (zero-length filament, NaN circulation, targets
    on a filament and its extension), and a wake whose trailing family has
    its ages shuffled (so only a few of its filaments still continue their
    neighbour), each forced onto the chained and the input-order layout and
    checked against the FP64 oracle."""
    g = load_golden("bs_edge.npz")
    fams = [(g["F1"], g["F2"], g["g"], g["rc"])]
    nt, nf = _count(g["P"].shape), _count(g["F1"].shape)
    for d in (1e-4, "visc2"):
        core, dv = wb.bs.parse_core(d)
        uo = g[f"u_oracle_{d if isinstance(d, str) else '0.0001'}_1000.0"]
        scale = np.abs(uo).max()
        for chained in (True, False):
            wb.set_tuning(core, nt, nf, 4, 64, 8.0)
            wb.set_layout(core, nt, nf, chained)
            u = wb.eval_host(fams, g["P"], core, dv, 1000.0, "f32c")
            assert wb.last_chained() == chained
            assert np.all(np.isfinite(u))
            assert np.abs(u - uo).max() <= F32C_TOL * scale, (d, chained)
    w = synth.make_wake(synth.RotorCase(nst=13, nsteps=40, dpsi_deg=6.0, seed=17))
    F1, F2 = synth.trail_filaments(w["dom"])
    perm = np.random.default_rng(3).permutation(F1.shape[2])  # shuffles the wake ages
    fams = [synth.shed_filaments(w["dom"]) + (w["gamma_shed"], w["rc_shed"]),
            (np.asfortranarray(F1[:, :, perm]), np.asfortranarray(F2[:, :, perm]),
             np.asfortranarray(w["gamma_trail"][:, :, perm]),
             np.asfortranarray(w["rc_trail"][:, :, perm]))]
    P = w["dom"]
    nt, nf = _count(P.shape), sum(_count(f[0].shape) for f in fams)
    uo = sum(oracle.c_eval(F1_, F2_, P, g_, rc_, "visc2", 1000.0) for F1_, F2_, g_, rc_ in fams)
    for chained in (True, False):
        wb.set_tuning(wb.bs.CORE_VATISTAS, nt, nf, 3, 64, 16.0)
        wb.set_layout(wb.bs.CORE_VATISTAS, nt, nf, chained)
        u = wb.eval_host(fams, P, wb.bs.CORE_VATISTAS, 2.0, 1000.0, "f32c")
        assert wb.last_chained() == chained
        assert per_target_rel(u, uo) < F32C_TOL, chained


def test_empty_inputs(wb, synth):
    w = synth.make_wake(synth.RotorCase(nst=5, nsteps=4))
    F1, F2 = synth.shed_filaments(w["dom"])
    u = wb.eval_host([], w["dom"], wb.bs.CORE_CUTOFF, 1e-4, 1000.0, "f32c")
    assert u.shape == w["dom"].shape and not u.any()
    e = np.zeros((0, 3, 1, 1), order="F")
    u = wb.eval_host([(F1, F2, w["gamma_shed"], w["rc_shed"])], e, wb.bs.CORE_CUTOFF, 1e-4, 1000.0)
    assert u.size == 0
    z = np.zeros((0, 3, 4, 3), order="F")
    u = wb.eval_host([(z, z, np.zeros((0, 1, 4, 3)), np.zeros((0, 1, 4, 3)))], w["dom"],
                     wb.bs.CORE_VATISTAS, 2.0, 1000.0)
    assert not u.any()


def test_mex_entry_on_gpu(wb, synth, ref):
    """BiotSavartMex through the library's mexFunction, as MATLAB calls it at
    WInDS.m:150 (cut-off, 'fuln') and with the Vatistas core ('visc', n=2)."""
    w = synth.make_wake(synth.RotorCase(nst=9, nsteps=12, seed=8))
    F1, F2 = synth.trail_filaments(w["dom"])
    hw = np.array([256.0, 1.0, 0.0])
    for d, cmod, dm in ((1e-4, "none", 1e-4), (2.0, "visc", "visc2")):
        for typ in ("fuln", "fuls", "full"):
            uind, L = wb.BiotSavartMex(F1, F2, w["dom"], w["gamma_trail"], w["rc_trail"], d, cmod,
                                       1000.0, typ, "true", hw)
            uo, _ = ref.biot_savart(F1, F2, w["dom"], w["gamma_trail"], w["rc_trail"], dm, 1000.0, "full")
            assert uind.shape == w["dom"].shape and not L.any()
            assert per_target_rel(uind, uo) < F32C_TOL
        # lifting-line points as P (core/KuttaJoukowski.m:216-219), 3-D P
        uind, _ = wb.BiotSavartMex(F1, F2, w["ll"], w["gamma_trail"], w["rc_trail"], d, cmod, 1000.0,
                                   "fuln", "false", hw)
        uo, _ = ref.biot_savart(F1, F2, w["ll"], w["gamma_trail"], w["rc_trail"], dm, 1000.0, "full")
        assert per_target_rel(uind, uo) < F32C_TOL


def test_biotsavart_api_2d_points(wb, synth, ref):
    w = synth.make_wake(synth.RotorCase(nst=6, nsteps=8, seed=9))
    F1, F2 = synth.shed_filaments(w["dom"])
    P2 = np.asfortranarray(synth.flat_points(w["dom"])[:17])  # [17, 3]
    u, L = wb.BiotSavart(F1, F2, P2, w["gamma_shed"], w["rc_shed"], "visc2", 1000.0, "full")
    uo, Lo = ref.biot_savart(F1, F2, P2, w["gamma_shed"], w["rc_shed"], "visc2", 1000.0, "full")
    assert u.shape == uo.shape
    np.testing.assert_allclose(L, Lo, rtol=1e-15)
    assert per_target_rel(u, uo) < F32C_TOL


def test_device_api_with_torch(wb, synth, oracle):
    import torch
    w = synth.make_wake(synth.RotorCase(nst=9, nsteps=20, seed=3))
    F1, F2 = synth.shed_filaments(w["dom"])
    dev = lambda a: torch.from_numpy(np.asarray(a).ravel(order="F").copy()).cuda()
    P = w["dom"]
    out = torch.zeros(P.size, dtype=torch.float64, device="cuda")
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        fam = (dev(F1), dev(F2), dev(w["gamma_shed"]), dev(w["rc_shed"]), F1.shape)
        wb.eval_device([fam], (dev(P), P.shape), wb.bs.CORE_VATISTAS, 2.0, 1000.0, out,
                       stream=s.cuda_stream)
    wb.sync(s.cuda_stream)
    u = out.cpu().numpy().reshape(P.shape, order="F")
    uo = oracle.c_eval(F1, F2, P, w["gamma_shed"], w["rc_shed"], "visc2", 1000.0)
    assert per_target_rel(u, uo) < F32C_TOL


def test_bounded_wait_timeout_is_reported(wb):
    """A bounded mbarrier wait with no producer runs out, the kernel returns,
    the host gets WINDS_BS_ERR_TIMEOUT, and the context stays usable."""
    rc = wb.lib().winds_bs_selftest_wait_timeout(C.c_ulonglong(2_000_000))
    assert rc == 3
    g = load_golden("bs_small_visc2.npz")
    u = wb.eval_host([(g["F1_shed"], g["F2_shed"], g["g_shed"], g["rc_shed"])], g["P_wake"],
                     wb.bs.CORE_VATISTAS, 2.0, 1000.0, "f32c")
    assert per_target_rel(u, g["u_oracle_shed_wake"]) < F32C_TOL


def test_fp32_peak_probe(wb):
    t = C.c_double()
    assert wb.lib().winds_bs_fp32_peak(C.byref(t)) == 0
    assert 20.0 < t.value < 200.0


def test_core_free_form(wb, oracle):
    """Targets far from every filament line (more than 54 core radii, the
    warp's ball included) take the core-free form for every pair, and match
    the FP64 oracle; targets inside the cores take it only for the far side
    of the ring. The same with the cut-off core. The counter reports exactly
    the pairs that took the form."""
    rng = np.random.default_rng(21)
    nf = 256
    a = np.linspace(0.0, 2 * np.pi, nf + 1)
    ring = np.stack([10.0 * np.cos(a), 10.0 * np.sin(a), 0.2 * np.sin(5 * a)], 1)
    F1 = np.asfortranarray(ring[:-1].reshape(nf, 3, 1, 1))
    F2 = np.asfortranarray(ring[1:].reshape(nf, 3, 1, 1))
    g = np.asfortranarray(rng.uniform(5.0, 15.0, (nf, 1, 1, 1)))
    rc = np.full((nf, 1, 1, 1), 0.01, order="F")  # squared core: rc = 0.1 m
    fams = [(F1, F2, g, rc)]
    # far: a small cloud 300 m above the ring (the lines lie in the ring's plane)
    Pf = np.asfortranarray((rng.uniform(-1.0, 1.0, (512, 3)) + [0.0, 0.0, 300.0]).reshape(512, 3, 1, 1))
    u = wb.eval_host(fams, Pf, wb.bs.CORE_VATISTAS, 2.0, 1000.0, "f32c")
    assert wb.last_core_free() == nf * 512
    uo = oracle.c_eval(F1, F2, Pf, g, rc, "visc2", 1000.0)
    # a closed ring seen from 30 radii away: its terms cancel to ~1/30 of
    # their size, which scales the FP32 rounding (the omitted core factor
    # differs from 1 by (0.1/300)^4 / 2 here)
    assert per_target_rel(u, uo) < F32C_TOL
    # near: targets on the ring, inside the cores of the nearby filaments
    Pn = np.asfortranarray((ring[:-1] + rng.normal(0.0, 0.05, (nf, 3))).reshape(nf, 3, 1, 1))
    u = wb.eval_host(fams, Pn, wb.bs.CORE_VATISTAS, 2.0, 1000.0, "f32c")
    uo = oracle.c_eval(F1, F2, Pn, g, rc, "visc2", 1000.0)
    assert per_target_rel(u, uo) < F32C_TOL
    assert wb.last_core_free() < nf * nf
    # cut-off: 300 m from 0.25 m segments with d = 1e-4, d |L|^2 is far below
    # FP32 resolution against r^4
    u = wb.eval_host(fams, Pf, wb.bs.CORE_CUTOFF, 1e-4, 1000.0, "f32c")
    assert wb.last_core_free() == nf * 512
    uo = oracle.c_eval(F1, F2, Pf, g, rc, 1e-4, 1000.0)
    assert per_target_rel(u, uo) < F32C_TOL
    u = wb.eval_host(fams, Pn, wb.bs.CORE_CUTOFF, 1e-4, 1000.0, "f32c")
    assert wb.last_core_free() < nf * nf
    uo = oracle.c_eval(F1, F2, Pn, g, rc, 1e-4, 1000.0)
    assert per_target_rel(u, uo) < F32C_TOL
