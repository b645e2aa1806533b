"""GPU parity of the blade kinematics (include/winds_kin.h) against the FP64
oracle (oracle/kin_ref.py: core/kinematics.m, core/velocity.m, DCMRot, ctdiff)
on a yawed, tilted, pre-coned rotor with pitch changes and platform motion."""
from __future__ import annotations

import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("motion,nb", [(False, 3), (True, 3), (True, 2)])
def test_kinematics_match_oracle(wb, synth, motion, nb):
    import kin_ref
    kin = importlib.import_module("winds-master_b200.kin")
    rc = synth.RotorCase(nst=13, nb=nb, nsteps=40, dpsi_deg=7.0, U=9.0)
    r = synth.rotor_series(rc, 37, pitch_deg=4.0, nac_yaw_deg=12.0, platform_motion=motion, seed=3)
    got = kin.kinematics(r)
    ref = kin_ref.kinematics(r)
    for key in ("hub", "lead", "quarter", "trail", "bound", "colloc", "end"):
        np.testing.assert_allclose(got[key], ref[key], rtol=0, atol=1e-11, err_msg=key)
    for key in ("bxt", "byt", "bzt", "bxn", "byn", "bzn"):
        np.testing.assert_allclose(got[key], ref[key], rtol=0, atol=1e-12, err_msg=key)
    # velocities come from differences of positions over dt: 1/dt amplifies ulps
    scale = np.abs(ref["vbound"]).max()
    for key in ("vbound", "vblade"):
        np.testing.assert_allclose(got[key], ref[key], rtol=0, atol=1e-10 * scale, err_msg=key)


def test_kinematics_feed_the_wake_step(wb, synth):
    """The device kinematics give the wake engine its quarter-chord and
    trailing-edge nodes and the lifting line its frames and inflow."""
    kin = importlib.import_module("winds-master_b200.kin")
    wake = importlib.import_module("winds-master_b200.wake")
    rc = synth.RotorCase(nst=9, nsteps=12, dpsi_deg=10.0, jitter=0.0)
    r = synth.rotor_series(rc, 8)
    k = kin.kinematics(r)
    c = synth.make_wake_case(rc, nsteps=8)
    c.update(quarter=k["quarter"], trailing=k["trail"])
    c["dom"][:, :, 0, :] = k["quarter"][:, :, 0, :]
    c["dom"][:, :, 1, :] = k["trail"][:, :, 0, :]
    b = wake.WakeBatch([c], integrator="pcc", precision="f64")
    b.step(3)
    st = b.state(0)
    np.testing.assert_array_equal(st["dom"][:, :, 0, :], k["quarter"][:, :, 3, :])
    np.testing.assert_array_equal(st["dom"][:, :, 1, :], k["trail"][:, :, 3, :])
    b.close()
