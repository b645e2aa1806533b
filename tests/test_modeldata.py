"""CPU tests of the rotor-model inputs (winds-master_b200/modeldata.py) on the
NREL 5-MW fixture made from the reference's model data."""
from __future__ import annotations

import importlib
import os

import numpy as np
import pytest

from conftest import GOLDEN


def _md():
    return importlib.import_module("winds-master_b200.modeldata")


def test_nrel_fixture_and_stations():
    md = _md()
    m = md.load_model(os.path.join(GOLDEN, "nrel5mw.npz"))
    assert len(m["r_trail"]) == 19 and m["r_trail"][0] == 1.5 and m["r_trail"][-1] == 63.0
    for t in m["tables"]:
        assert np.all(np.diff(t["aoa"]) > 0) and t["aoa"][0] == -180.0 and t["aoa"][-1] == 180.0
    st = md.stations(m["r_trail"], m["chord_trail"], m["twist_trail"], m["nfoil_trail"])
    assert len(st["r_nodes"]) == 18
    np.testing.assert_allclose(st["dr"].sum(), 63.0 - 1.5)
    # nearest airfoil of each station, ties to the outer node
    rt = m["r_trail"]
    for i, rn in enumerate(st["r_nodes"]):
        j = i if rn - rt[i] < rt[i + 1] - rn else i + 1
        assert st["nfoil"][i] == m["nfoil_trail"][j]
    # root stations carry the cylinders (Cl = 0)
    assert m["names"][st["nfoil"][0] - 1].startswith("Cylinder")
    assert np.all(m["tables"][0]["cl"] == 0.0)


REF_TREE = os.environ.get("WINDS_REFERENCE", "")


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF_TREE, "modeldata")) or not REF_TREE,
                    reason="reference tree not given (WINDS_REFERENCE)")
def test_fixture_regenerates_from_reference(tmp_path):
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_nrel", os.path.join(GOLDEN, "make_nrel.py"))
    mk = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mk)
    d0 = dict(np.load(os.path.join(GOLDEN, "nrel5mw.npz")))
    cwd = os.getcwd()
    try:
        mk.main(REF_TREE)
    finally:
        os.chdir(cwd)
    d1 = dict(np.load(os.path.join(GOLDEN, "nrel5mw.npz")))
    assert d0.keys() == d1.keys()
    for k in d0:
        np.testing.assert_array_equal(d0[k], d1[k])


def test_nrel_oracle_step_is_plausible():
    """One step of the FP64 oracle chain on the NREL rotor at 11.4 m/s, TSR 7:
    the lifting line converges and the rotor thrust is of the rated order."""
    import kin_ref
    import kj_ref
    import wake_ref
    md = _md()
    m = md.load_model(os.path.join(GOLDEN, "nrel5mw.npz"))
    ser = md.operating_series(m, nsteps=6, na=20)
    wc, kj = md.cases(m, ser, kin_ref.kinematics(ser))
    r = kj_ref.KJWakeRef(wake_ref.WakeCaseRef(**{k: wc[k] for k in wake_ref.WakeCaseRef.__dataclass_fields__}),
                         kj, integrator="pcc", relax=0.25, tol=1e-6, maxiter=200, d=1e-4)
    r.step()
    assert r.kj_iters < 200
    assert 2e5 < r.T < 1.5e6 and r.P > 0


def _fast_channels(m, nsteps=30, na=12):
    """FAST-style channels of a yawed rotor on a pitching platform."""
    md = _md()
    ser = md.operating_series(m, U=10.0, tsr=7.5, pitch=2.0, yaw=8.0, nsteps=nsteps, na=na)
    t = ser["time"]
    ch = {"Time": t, "Azimuth": ser["azimuth"]}
    for b in range(int(m["nb"])):
        ch[f"BldPitch{b + 1}"] = ser["pitch"][:, b] + 0.5 * np.sin(0.3 * t + b)
    ch["NacYaw"] = ser["nac_yaw"]
    names = ("PtfmSurge", "PtfmSway", "PtfmHeave", "PtfmRoll", "PtfmPitch", "PtfmYaw")
    amp = (0.4, 0.1, 0.05, 0.3, 1.2, 0.2)
    for k, (n, a) in enumerate(zip(names, amp)):
        ch[n] = a * np.sin(0.2 * t + k)
    ch["WindVxi"], ch["WindVyi"], ch["WindVzi"] = ser["wind"][:, 0], ser["wind"][:, 1], ser["wind"][:, 2]
    ch["RotSpeed"] = np.full_like(t, ser["_omega"] * 30.0 / np.pi)
    return ser, ch


def test_fast_out_roundtrip_and_resampling(tmp_path):
    """output_import.m's reading: names on line 7, units on 8, samples after;
    channels interpolated linearly to t0:1/freq:t1, clamped to the record."""
    md = _md()
    m = md.load_model(os.path.join(GOLDEN, "nrel5mw.npz"))
    _, ch = _fast_channels(m)
    path = str(tmp_path / "run.out")
    md.write_fast_out(path, ch)
    fo = md.read_fast_out(path)
    assert fo["units"]["Time"] == "(s)" and fo["units"]["Azimuth"] == "(deg)"
    for k, v in ch.items():
        np.testing.assert_allclose(fo[k], v, rtol=1e-9, atol=1e-9)
    t = ch["Time"]
    t0, t1, freq = float(t[2]) + 0.03, float(t[-3]), 25.0
    fr = md.read_fast_out(path, (t0, t1, freq))
    ti = t0 + np.arange(int(np.floor((t1 - t0) * freq + 1e-9)) + 1) / freq
    np.testing.assert_allclose(fr["Time"], ti, rtol=0, atol=1e-12)
    for k in ("Azimuth", "PtfmPitch", "BldPitch2"):
        np.testing.assert_allclose(fr[k], np.interp(ti, fo["Time"], fo[k]), rtol=1e-12, atol=1e-12)
    fc = md.read_fast_out(path, (float(t[0]) - 5.0, float(t[-1]) + 5.0, 0.0))
    assert fc["Time"][0] == fo["Time"][0] and abs(fc["Time"][-1] - fo["Time"][-1]) < 1e-9


def test_series_from_fastout_matches_kinematics(tmp_path):
    """A FAST time series through series_from_fastout gives the same blade
    kinematics (FP64 oracle) as the series it was written from."""
    import kin_ref
    md = _md()
    m = md.load_model(os.path.join(GOLDEN, "nrel5mw.npz"))
    ser, ch = _fast_channels(m)
    ser = dict(ser, pitch=np.stack([ch[f"BldPitch{b + 1}"] for b in range(int(m["nb"]))], 1),
               ptfm=np.stack([ch[n] for n in ("PtfmSurge", "PtfmSway", "PtfmHeave", "PtfmRoll",
                                              "PtfmPitch", "PtfmYaw")], 1))
    path = str(tmp_path / "run.out")
    md.write_fast_out(path, ch)
    fs = md.series_from_fastout(m, md.read_fast_out(path), na=12)
    k0, k1 = kin_ref.kinematics(ser), kin_ref.kinematics(fs)
    for name in ("quarter", "trail", "bound", "bxn", "vblade"):
        np.testing.assert_allclose(k1[name], k0[name], rtol=1e-8, atol=1e-8)
    wc, kj = md.cases(m, fs, k1)
    assert wc["nsteps"] == fs["_nsteps"] + 1 and kj["rpm"].shape == (wc["nsteps"],)
    np.testing.assert_allclose(kj["rpm"], ch["RotSpeed"][11:], rtol=1e-9)  # 11 digits written
    # blade pitch per step and blade for the loads; the twist is the aerodynamic twist alone
    assert kj["pitch"].shape == (wc["nsteps"], int(m["nb"]))
    np.testing.assert_allclose(kj["pitch"][:, 1], ch["BldPitch2"][11:], rtol=1e-9, atol=1e-9)
    st = md.stations(m["r_trail"], m["chord_trail"], m["twist_trail"], m["nfoil_trail"])
    np.testing.assert_allclose(kj["twist"], np.radians(st["twist"]), rtol=1e-15)


def test_fast_out_regrids_time_with_the_integration_step(tmp_path):
    """output_import.m:44-46: for a non-Simulink run the time column is
    rebuilt as t_first:dt:t_last from the .fst integration step."""
    md = _md()
    t = np.array([0.0, 0.0999, 0.2001, 0.3, 0.4])  # rounded times as a file may hold them
    ch = {"Time": t, "Azimuth": 90.0 * t}
    path = str(tmp_path / "run.out")
    md.write_fast_out(path, ch)
    fo = md.read_fast_out(path, dt=0.1)
    np.testing.assert_allclose(fo["Time"], 0.1 * np.arange(5), rtol=0, atol=1e-12)
    np.testing.assert_allclose(fo["Azimuth"], 90.0 * t, rtol=1e-9)
