"""CPU tests of the kinematics oracle (oracle/kin_ref.py): the rotation
conventions of core/DCMRot.m and core/kinematics.m, ctdiff's stencils, and
the blade frames of core/velocity.m."""
from __future__ import annotations

import numpy as np


def test_dcm_conventions_and_exact_quadrants():
    import kin_ref
    # multiples of 90 degrees are exact, as MATLAB's sind/cosd
    s, c = kin_ref.sincosd(np.array([0.0, 90.0, 180.0, 270.0, -90.0, 450.0]))
    np.testing.assert_array_equal(s, [0.0, 1.0, 0.0, -1.0, -1.0, 1.0])
    np.testing.assert_array_equal(np.abs(c), [1.0, 0.0, 1.0, 0.0, 0.0, 0.0])
    # Rz(90) maps x to y (DCMRot.m:35); a sequence applies its first rotation first
    A = kin_ref.dcm(np.array([90.0]), "z")
    np.testing.assert_allclose(kin_ref.apply(A, np.array([1.0, 0.0, 0.0])), [0.0, 1.0, 0.0], atol=1e-15)
    A = kin_ref.dcm(np.array([90.0, 90.0]), "zx")
    np.testing.assert_allclose(kin_ref.apply(A, np.array([1.0, 0.0, 0.0])), [0.0, 0.0, 1.0], atol=1e-15)
    rng = np.random.default_rng(0)
    A = kin_ref.dcm(rng.uniform(-180, 180, (20, 11)), kin_ref.SEQ_ROTOR)
    np.testing.assert_allclose(A @ np.swapaxes(A, -1, -2), np.broadcast_to(np.eye(3), A.shape), atol=1e-14)
    np.testing.assert_allclose(np.linalg.det(A), 1.0, atol=1e-14)


def test_ctdiff_exact_for_quadratics():
    import kin_ref
    t = 0.1 * np.arange(12)
    y = 3.0 * t ** 2 - 2.0 * t + 1.0
    np.testing.assert_allclose(kin_ref.ctdiff(t, y[:, None], 0)[:, 0], 6.0 * t - 2.0, atol=1e-12)


def test_rotor_at_rest_geometry_and_frames(synth):
    import kin_ref
    rc = synth.RotorCase(nst=9, nsteps=20, dpsi_deg=10.0)
    r = synth.rotor_series(rc, 8, tilt_deg=0.0, precone_deg=0.0)
    r.update(azimuth=np.zeros(8), pitch=np.zeros((8, 3)), overhang=0.0, twr2shft=0.0)
    k = kin_ref.kinematics(r)
    hub = np.array([0.0, 0.0, r["tower_ht"]])
    np.testing.assert_allclose(k["hub"], np.broadcast_to(hub, (8, 3)), atol=1e-12)
    # blade 1 at azimuth 0 points up (+z); twist turns the chord about the span
    q = k["quarter"][:, :, 0, 0]
    np.testing.assert_allclose(q - hub, np.stack([0 * r["r_trail"], 0 * r["r_trail"], r["r_trail"]], 1), atol=1e-12)
    tw = np.radians(r["twist_trail"])
    te = k["trail"][:, :, 0, 0] - q
    c = 0.75 * r["chord_trail"]
    np.testing.assert_allclose(te[:, 0], -c * np.sin(tw), atol=1e-12)   # Rz(twist + 90) of (c, 0, 0)
    np.testing.assert_allclose(te[:, 1], c * np.cos(tw), atol=1e-12)
    # blades 120 degrees apart about x
    q2 = k["quarter"][:, :, 0, 1] - hub
    np.testing.assert_allclose(q2[:, 2], r["r_trail"] * np.cos(np.radians(120.0)), atol=1e-12)
    # frames: unit, orthogonal, right-handed; vel.blade of a rotor at rest is the wind
    bx, by, bz = k["bxn"], k["byn"], k["bzn"]
    np.testing.assert_allclose((bx * bz).sum(1), 0.0, atol=1e-12)
    np.testing.assert_allclose((by * by).sum(1), 1.0, atol=1e-12)
    np.testing.assert_allclose(np.linalg.norm(k["vbound"], axis=1), rc.U, rtol=1e-12)
