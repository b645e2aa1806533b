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


def test_fast_series_on_a_moving_platform(wb, tmp_path):
    """The same chain from a FAST output file (modeldata.read_fast_out, the
    layout of core/output_import.m): a pitching, surging platform, blade
    pitch varying per blade and time, 8 deg yaw, through device kinematics
    and two pcc steps with the lifting line and loads, against the oracle chain."""
    import kin_ref
    import kj_ref
    import wake_ref
    md = importlib.import_module("winds-master_b200.modeldata")
    kin = importlib.import_module("winds-master_b200.kin")
    wake = importlib.import_module("winds-master_b200.wake")
    m = md.load_model(os.path.join(GOLDEN, "nrel5mw.npz"))
    ser = md.operating_series(m, U=10.0, tsr=7.5, pitch=2.0, yaw=8.0, nsteps=6, na=24)
    t = ser["time"]
    ch = {"Time": t, "Azimuth": ser["azimuth"]}
    for b in range(int(m["nb"])):
        ch[f"BldPitch{b + 1}"] = ser["pitch"][:, b] + 0.5 * np.sin(0.3 * t + b)
    ch["NacYaw"] = ser["nac_yaw"]
    for k, (n, a) in enumerate(zip(("PtfmSurge", "PtfmSway", "PtfmHeave", "PtfmRoll", "PtfmPitch",
                                    "PtfmYaw"), (0.4, 0.1, 0.05, 0.3, 1.2, 0.2))):
        ch[n] = a * np.sin(0.2 * t + k)
    ch["WindVxi"], ch["WindVyi"], ch["WindVzi"] = ser["wind"][:, 0], ser["wind"][:, 1], ser["wind"][:, 2]
    ch["RotSpeed"] = np.full_like(t, ser["_omega"] * 30.0 / np.pi)
    path = str(tmp_path / "run.out")
    md.write_fast_out(path, ch)
    fs = md.series_from_fastout(m, md.read_fast_out(path), na=24)
    wc, kj = md.cases(m, fs, kin.kinematics(fs))
    wr, kr = md.cases(m, fs, kin_ref.kinematics(fs))
    b = wake.WakeBatch([wc], integrator="pcc", d=1e-4, precision="f32c")
    b.set_kj([kj], relax=0.25, tol=1e-6, maxiter=200)
    r = kj_ref.KJWakeRef(wake_ref.WakeCaseRef(**{k: wr[k] for k in wake_ref.WakeCaseRef.__dataclass_fields__}),
                         kr, integrator="pcc", relax=0.25, tol=1e-6, maxiter=200, d=1e-4)
    for step in range(2):
        b.step(1, graph=True)
        r.step()
        T, _, P = b.loads()
        assert abs(T[0] - r.T) <= 1e-4 * abs(r.T), (step, T[0], r.T)
        assert abs(P[0] - r.P) <= 1e-4 * abs(r.P), (step, P[0], r.P)
        np.testing.assert_allclose(b.bound(0), r.bound, rtol=0, atol=1e-4 * np.abs(r.bound).max())
    b.close()
