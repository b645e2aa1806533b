"""End to end on the NREL 5-MW rotor (model data of the reference, fixture
tests/golden/nrel5mw.npz): device kinematics, pcc wake steps, the lifting-line
iteration and rotor loads against the FP64 oracle chain (kinematics.m /
velocity.m, the step, kj(), perform.m) at 11.4 m/s, TSR 7, 10 deg nacelle
yaw, the reference's defaults (cut-off core d = 1e-4, relax 0.25)."""
from __future__ import annotations

import importlib
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", ["f64", "f32c"])
def test_nrel_run_matches_oracle(wb, prec):
    import kin_ref
    import kj_ref
    import wake_ref
    md = importlib.import_module("winds-master_b200.modeldata")
    kin = importlib.import_module("winds-master_b200.kin")
    wake = importlib.import_module("winds-master_b200.wake")
    m = md.load_model(os.path.join(GOLDEN, "nrel5mw.npz"))
    ser = md.operating_series(m, nsteps=6, na=30, yaw=10.0)
    wc, kj = md.cases(m, ser, kin.kinematics(ser))
    wr, kr = md.cases(m, ser, kin_ref.kinematics(ser))
    b = wake.WakeBatch([wc], integrator="pcc", d=1e-4, precision=prec)
    b.set_kj([kj], relax=0.25, tol=1e-6, maxiter=200)
    r = kj_ref.KJWakeRef(wake_ref.WakeCaseRef(**{k: wr[k] for k in wake_ref.WakeCaseRef.__dataclass_fields__}),
                         kr, integrator="pcc", relax=0.25, tol=1e-6, maxiter=200, d=1e-4)
    for step in range(4):
        b.step(1)
        r.step()
        it = int(b.kj_stats()[0][0])
        T, _, P = b.loads()
        g = b.bound(0)
        scale = np.abs(r.bound).max()
        assert it < 200 and r.kj_iters < 200
        assert abs(it - r.kj_iters) <= 1, (step, it, r.kj_iters)
        tol = 1e-8 if prec == "f64" else 1e-4
        np.testing.assert_allclose(g, r.bound, rtol=0, atol=tol * scale)
        assert abs(T[0] - r.T) <= 1e-4 * abs(r.T), (step, T[0], r.T)
        assert abs(P[0] - r.P) <= 1e-4 * abs(r.P), (step, P[0], r.P)
    b.close()
