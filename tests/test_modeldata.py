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


@pytest.mark.skipif(not os.path.isdir("/root/reference/modeldata"), reason="reference tree absent")
def test_fixture_regenerates_from_reference(tmp_path):
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_nrel", os.path.join(GOLDEN, "make_nrel.py"))
    mk = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mk)
    d0 = dict(np.load(os.path.join(GOLDEN, "nrel5mw.npz")))
    cwd = os.getcwd()
    try:
        mk.main("/root/reference")
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
