"""GPU parity of the device Kutta-Joukowski fixed point (winds_wake_set_kj)
against the FP64 oracle (oracle/kj_ref.py: the step oracle with
core/KuttaJoukowski.m's 'fixed' loop), two uneven cases per batch."""
from __future__ import annotations

import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cases(synth):
    ra = synth.RotorCase(nst=9, nsteps=14, dpsi_deg=8.0, seed=21, jitter=0.0)
    rb = synth.RotorCase(nst=6, nb=2, nsteps=22, dpsi_deg=6.0, U=8.0, yaw_deg=20.0, shear=0.2, seed=22)
    out = []
    for r in (ra, rb):
        c = synth.make_wake_case(r, nsteps=10, jitter=0.02)
        out.append((c, synth.make_kj_case(r, nsteps=c["nsteps"], t0=c["t0"])))
    return out


def _refs(cases, **kw):
    import kj_ref
    import wake_ref
    return [kj_ref.KJWakeRef(wake_ref.WakeCaseRef(**{k: c[k] for k in wake_ref.WakeCaseRef.__dataclass_fields__}),
                             kj, **kw) for c, kj in cases]


@pytest.mark.parametrize("prec", ["f64", "f32c"])
def test_kj_step_matches_oracle(wb, synth, prec):
    wake = importlib.import_module("winds-master_b200.wake")
    cases = _cases(synth)
    tol, relax, maxiter = 1e-4, 0.3, 25
    batch = wake.WakeBatch([c for c, _ in cases], integrator="pcc", precision=prec)
    batch.set_kj([k for _, k in cases], relax=relax, tol=tol, maxiter=maxiter)
    refs = _refs(cases, integrator="pcc", relax=relax, tol=tol, maxiter=maxiter)
    for step in range(3):
        batch.step(1)
        iters, res, nev = batch.kj_stats()
        T, Q, P = batch.loads()
        for k, r in enumerate(refs):
            r.step()
            st = batch.state(k)
            cl, cd, aoa = batch.perf(k)
            scale = np.abs(r.bound).max()
            if prec == "f64":
                # identical iteration; sums in another order than the oracle's
                assert iters[k] == r.kj_iters, (step, k, iters[k], r.kj_iters)
                np.testing.assert_allclose(st["bound"], r.bound, rtol=0, atol=1e-9 * scale)
                np.testing.assert_allclose(aoa, r.aoa, rtol=0, atol=1e-8)
                np.testing.assert_allclose(cl, r.cl, rtol=0, atol=1e-9)
                np.testing.assert_allclose(cd, r.cd, rtol=0, atol=1e-9)
                assert abs(res[k] - r.kj_res) <= 1e-8 * max(r.kj_res, 1e-12) + 1e-14
            else:
                # FP32 induced velocity at 1e-6 relative: the converged Γ agrees
                # to the tolerance's order, the iteration count within one
                assert abs(int(iters[k]) - r.kj_iters) <= 1, (step, k, iters[k], r.kj_iters)
                np.testing.assert_allclose(st["bound"], r.bound, rtol=0, atol=5 * tol * scale)
                np.testing.assert_allclose(aoa, r.aoa, rtol=0, atol=1e-3)
            # rotor loads of the step (postproc/perform.m) at the run tolerance
            import perform_ref
            Td, Qd, Pd, _ = perform_ref.loads(cl, cd, aoa, cases[k][1]["vblade"][:, :, step, :],
                                             np.degrees(cases[k][1]["twist"]), cases[k][1]["chord"],
                                             cases[k][1]["r_station"], cases[k][1]["dr_station"],
                                             cases[k][1]["rpm"][step], cases[k][1]["rho"])
            # the device formula on the device's own Cl, Cd, AoA: same arithmetic
            assert abs(T[k] - Td) <= 1e-9 * abs(Td) and abs(P[k] - Pd) <= 1e-9 * abs(Pd)
            assert abs(T[k] - r.T) <= 1e-4 * abs(r.T) and abs(P[k] - r.P) <= 1e-4 * abs(r.P), (T[k], r.T, P[k], r.P)
            # the step's Γ is re-formed from the converged bound (kj(), :285-288)
            np.testing.assert_allclose(st["shed"][:, 0], st["bound"], rtol=0, atol=0)
            # carrying the state on: compare on the oracle's own trajectory
            r.bound = st["bound"].copy()
        assert nev == int(iters.max())


@pytest.mark.parametrize("maxiter", [25, 2])
def test_kj_graph_replay_is_bit_identical(wb, synth, maxiter):
    """The graph path runs each step as one graph whose lifting-line
    iteration is a conditional WHILE node (no host round trip per iteration);
    it must give the host-driven loop's results bit for bit, including the
    iteration counts and the stop at maxiter."""
    wake = importlib.import_module("winds-master_b200.wake")
    cases = _cases(synth)
    out = []
    for graph in (False, True):
        b = wake.WakeBatch([c for c, _ in cases], integrator="pcc")
        b.set_kj([k for _, k in cases], relax=0.3, tol=1e-4, maxiter=maxiter)
        rec = []
        for _ in range(3):
            b.step(1, graph=graph)
            iters, res, nev = b.kj_stats()
            rec.append((iters.copy(), res.copy(), nev, b.loads()))
        out.append(([b.state(k) for k in range(2)], rec))
        b.close()
    for k in range(2):
        for key in ("dom", "bound", "shed", "trail"):
            np.testing.assert_array_equal(out[0][0][k][key], out[1][0][k][key])
    for (i0, r0, n0, l0), (i1, r1, n1, l1) in zip(out[0][1], out[1][1]):
        np.testing.assert_array_equal(i0, i1)
        np.testing.assert_array_equal(r0, r1)
        assert n0 == n1 and n0 == i0.max() and n0 <= maxiter
        for a, c in zip(l0, l1):
            np.testing.assert_array_equal(a, c)
    if maxiter == 2:
        assert all((r[0] == 2).all() for r in out[1][1])


@pytest.mark.parametrize("graph", [False, True])
def test_kj_diverged_reports_error(wb, synth, graph):
    """An angle of attack outside the airfoil table gives NaN Cl; the solver
    stops with the reference's 'Diverging soln!!!' as an error code."""
    wake = importlib.import_module("winds-master_b200.wake")
    bs = importlib.import_module("winds-master_b200.bs")
    cases = _cases(synth)
    kjs = []
    for _, kj in cases:
        kj = dict(kj)
        sel = np.abs(kj["aoa"]) <= 0.5  # table covers only [-0.5, 0.5] deg
        kj.update(aoa=kj["aoa"][sel], cl=kj["cl"][sel], cd=kj["cd"][sel],
                  foil_points=np.array([sel.sum()], dtype=np.int32))
        kjs.append(kj)
    b = wake.WakeBatch([c for c, _ in cases], integrator="fe", precision="f64")
    b.set_kj(kjs, relax=0.3, tol=1e-4, maxiter=5)
    with pytest.raises(bs.WindsError) as ei:
        b.step(1, graph=graph)
    assert ei.value.code == 6
    # the context stays usable
    b.close()
    b2 = wake.WakeBatch([c for c, _ in cases], integrator="fe", precision="f64")
    b2.step(1)
    b2.close()
