"""CPU tests of the free-wake step oracle (oracle/wake_ref.py) on properties
the reference's step must have."""
from __future__ import annotations

import numpy as np
import pytest


@pytest.fixture(scope="module")
def wake_ref():
    import wake_ref as w
    return w


def _case(synth, wake_ref, gamma_zero=False, **kw):
    rc = synth.RotorCase(nst=6, nsteps=9, dpsi_deg=10.0, seed=3, **kw)
    c = synth.make_wake_case(rc, nsteps=8)
    if gamma_zero:
        c["bound"][:] = 0.0
        c["trail_gamma"][:] = 0.0
    return wake_ref.WakeCaseRef(**{k: c[k] for k in wake_ref.WakeCaseRef.__dataclass_fields__})


@pytest.mark.parametrize("integ", ["fe", "ab2", "ab4", "pcc"])
def test_zero_circulation_convects_with_freestream(synth, wake_ref, integ):
    """No vorticity: every integrator moves the wake rigidly with the wind,
    except where ab2/ab4 pad the shifted velocity history with zeros
    (ab2.m:39, ab4.m:79-81: the youngest columns)."""
    c = _case(synth, wake_ref, gamma_zero=True)
    w = wake_ref.WakeRef(c, integrator=integ)
    first = {"fe": 2, "pcc": 2, "ab2": 3, "ab4": 5}[integ]
    for _ in range(4):
        before = w.dom.copy()
        w.step()
        assert np.abs(w.uind).max() == 0.0
        np.testing.assert_allclose(w.dom[:, :, first:], before[:, :, first - 1:-1] + c.dt * np.array(
            [c.wind[0, 0], 0.0, 0.0])[None, :, None, None], rtol=0, atol=1e-12)
        np.testing.assert_array_equal(w.dom[:, :, 0], c.quarter[:, :, w.step_idx])


def test_bookkeeping_conserves_circulation(synth, wake_ref):
    """Kelvin: every trailing column sums to zero across the span and the shed
    columns close the trailing ones (WInDS.m:131-140)."""
    c = _case(synth, wake_ref)
    shed, trail = wake_ref.bookkeeping(c.bound, c.trail_gamma)
    np.testing.assert_allclose(trail.sum(axis=0), 0.0, atol=1e-11)
    np.testing.assert_allclose(shed[:, 1:].sum(axis=1) + trail[:-1].cumsum(axis=0)[:, 0], 0.0,
                               atol=1e-10)
    np.testing.assert_array_equal(shed[:, 0], c.bound)


def test_rigid_translation_has_no_stretch(synth, wake_ref):
    c = _case(synth, wake_ref)
    sh, tr = wake_ref.lengths(c.dom)
    moved = c.dom + np.array([1.5, -0.5, 2.0])[None, :, None, None]
    sh2, tr2 = wake_ref.lengths(moved)
    shed, trail = wake_ref.bookkeeping(c.bound, c.trail_gamma)
    a = wake_ref.cores(c, shed, trail, 0.0, (sh2, tr2), (sh, tr), True)
    b = wake_ref.cores(c, shed, trail, 0.0, (sh, tr), None, False)
    for x, y in zip(a, b):
        np.testing.assert_allclose(x, y, rtol=1e-12)


def test_core_growth_formula(synth, wake_ref):
    """Age form rc^2 = rc0^2 + 4 alpha delta nu (1 + a1 Re) age; vcore.m form
    r0^2 + 4 alpha nu (1 + a1 Re) t."""
    c = _case(synth, wake_ref)
    g = np.array([0.0, 3.0, -7.0])
    age = np.array([0.0, 0.5, 2.0])
    np.testing.assert_allclose(wake_ref.core(c, g, age),
                               c.rc0 ** 2 + 4 * c.alpha * c.delta * c.nu * (1 + c.a1 * np.abs(g) / c.nu) * age)
    c.core_mode = 0
    np.testing.assert_allclose(wake_ref.core(c, g, 1.5),
                               c.r0 ** 2 + 4 * c.alpha * c.nu * (1 + c.a1 * np.abs(g) / c.nu) * 1.5)


def test_kj_oracle_interp1_is_nan_outside():
    import kj_ref
    x = np.array([-2.0, 0.0, 3.0])
    y = np.array([1.0, 2.0, 5.0])
    out = kj_ref.interp1(x, y, np.array([-3.0, -1.0, 1.5, 3.0, 4.0, np.nan]))
    assert np.isnan(out[0]) and np.isnan(out[4]) and np.isnan(out[5])
    np.testing.assert_allclose(out[1:4], [1.5, 3.5, 5.0])


def test_kj_oracle_fixed_point(synth):
    """The fixed point contracts and leaves the shed column equal to the
    converged bound circulation (core/KuttaJoukowski.m:42-49, kj() :277-290)."""
    import kj_ref
    import wake_ref
    r = synth.RotorCase(nst=7, nsteps=8, dpsi_deg=10.0, seed=5, jitter=0.0)
    c = synth.make_wake_case(r, nsteps=6)
    kj = synth.make_kj_case(r, nsteps=c["nsteps"], t0=c["t0"])
    ref = kj_ref.KJWakeRef(wake_ref.WakeCaseRef(**{k: c[k] for k in wake_ref.WakeCaseRef.__dataclass_fields__}),
                           kj, relax=0.3, tol=1e-5, maxiter=60)
    ref.step()
    assert ref.kj_iters < 60 and ref.kj_res <= 1e-5
    np.testing.assert_array_equal(ref.shed[:, 0], ref.bound)
    np.testing.assert_allclose(ref.trail[:, 0].sum(0), 0.0, atol=1e-12)
    # a table too narrow for the flow's angle of attack diverges
    bad = dict(kj, aoa=np.array([-0.5, 0.5]), cl=np.array([0.0, 0.1]), cd=np.array([0.01, 0.01]),
               foil_points=np.array([2], dtype=np.int32))
    with pytest.raises(kj_ref.KJDiverged):
        kj_ref.kj_solve(bad, 0, c["dom"], ref.trail_prev, ref.rcs, ref.rct, ref.bound)


def test_perform_oracle_rotation_and_totals():
    """perform.m's 'zzz' DCMRot sequence [-90, twist, pitch] equals one z
    rotation by twist + pitch - 90 (core/DCMRot.m:27-45); totals sum every
    station and blade; a station with zero Cl and Cd carries no load."""
    import perform_ref

    def dcm(seq_deg):  # DCMRot: A <- R A for each rotation, y = A x
        A = np.eye(3)
        for t in seq_deg:
            A = perform_ref.rz(t) @ A
        return A

    for tw, pitch in ((5.0, 2.0), (-3.0, 17.5), (13.0, 0.0)):
        np.testing.assert_allclose(dcm([-90.0, tw, pitch]), perform_ref.rz(tw + pitch - 90.0), atol=1e-15)
    rng = np.random.default_rng(0)
    ns, nb = 5, 3
    vb = rng.normal(0, 1, (ns, 3, nb)) + np.array([[[-9.0], [-40.0], [0.0]]])
    cl, cd, aoa = rng.uniform(0.2, 1.2, (ns, nb)), rng.uniform(0.01, 0.05, (ns, nb)), rng.uniform(2, 10, (ns, nb))
    th = rng.uniform(0, 10, ns)
    chord, r, dr = np.full(ns, 2.0), np.linspace(10, 60, ns), np.full(ns, 10.0)
    T, Q, P, dT = perform_ref.loads(cl, cd, aoa, vb, th, chord, r, dr, 12.1, 1.225)
    assert abs(T - dT.sum()) < 1e-9 * abs(T)
    assert abs(P - np.pi / 30 * 12.1 * Q) < 1e-9 * abs(P)
    cl[2, 1] = cd[2, 1] = 0.0
    _, _, _, dT0 = perform_ref.loads(cl, cd, aoa, vb, th, chord, r, dr, 12.1, 1.225)
    assert dT0[2, 1] == 0.0


def test_perform_pitch_per_blade_matches_blade_by_blade():
    """perform.m:22-33 rotates and subtracts twist + BldPitch<b> per blade:
    the loads with a [ns, nb] angle equal the sum of single-blade loads."""
    import perform_ref
    rng = np.random.default_rng(4)
    ns, nb = 9, 3
    cl, cd = rng.uniform(0.2, 1.2, (ns, nb)), rng.uniform(0.01, 0.05, (ns, nb))
    aoa = rng.uniform(2.0, 10.0, (ns, nb))
    vb = np.stack([rng.uniform(-10, -5, (ns, nb)), rng.uniform(40, 60, (ns, nb)),
                   rng.uniform(-1, 1, (ns, nb))], 1)
    twist = rng.uniform(0.0, 13.0, ns)
    pitch = rng.uniform(0.0, 8.0, nb)
    chord, r, dr = rng.uniform(1.5, 4.0, ns), np.linspace(5, 60, ns), np.full(ns, 6.0)
    T, Q, P, dT = perform_ref.loads(cl, cd, aoa, vb, twist[:, None] + pitch[None, :], chord, r, dr,
                                    12.1, 1.225)
    tot = np.zeros(3)
    for b in range(nb):
        t1, q1, p1, d1 = perform_ref.loads(cl[:, b:b + 1], cd[:, b:b + 1], aoa[:, b:b + 1],
                                           vb[:, :, b:b + 1], twist + pitch[b], chord, r, dr, 12.1, 1.225)
        tot += (t1, q1, p1)
        np.testing.assert_allclose(dT[:, b], d1[:, 0], rtol=1e-14)
    np.testing.assert_allclose((T, Q, P), tot, rtol=1e-12)
