"""Inputs of a WInDS run from its initial state on the NREL 5-MW rotor
(fixture tests/golden/nrel5mw.npz), for the literal oracle of the driver loop
(oracle/winds_ref.py) and the device engine: the reference's defaults
(cut-off core d = 1e-4, co = 1000, relax 0.25, maxiter 30, 10 Hz) with a
gusting wind, 10 deg nacelle yaw and a recorded tip-speed ratio that varies
from step to step (fastout.TipSpdRat, so wake.r0 changes every step)."""
from __future__ import annotations

import importlib
import os

import numpy as np

from conftest import GOLDEN


def nrel_series(nsteps=31, U=11.4, tsr=7.0, yaw=10.0, gust=0.4):
    md = importlib.import_module("winds-master_b200.modeldata")
    m = md.load_model(os.path.join(GOLDEN, "nrel5mw.npz"))
    ser = md.operating_series(m, U=U, tsr=tsr, yaw=yaw, nsteps=nsteps, na=1)
    t = ser["time"]
    ser["wind"][:, 0] = U + gust * np.sin(0.7 * t)
    ser["tsr"] = tsr * (1.0 + 0.05 * np.sin(0.9 * t))
    return m, ser


def cl0_geometric(m, ser, kin):
    """Stand-in for BEM's Cl at time index 1 (core/initials.m:116): each
    station's table at the blade-frame inflow angle without induction."""
    md = importlib.import_module("winds-master_b200.modeldata")
    st = md.stations(m["r_trail"], m["chord_trail"], m["twist_trail"], m["nfoil_trail"])
    vb = kin["vblade"][:, :, 0, 0]
    aoa = np.degrees(np.arctan2(-vb[:, 1], vb[:, 0]))
    return np.array([np.interp(aoa[i], m["tables"][f - 1]["aoa"], m["tables"][f - 1]["cl"])
                     for i, f in enumerate(st["nfoil"])])


def oracle_run(m, ser, kin, cl0, integ="pcc", tol=1e-8, maxiter=30, relax=0.25, d=1e-4, co=1000.0,
               rho=1.23):
    import winds_ref
    md = importlib.import_module("winds-master_b200.modeldata")
    st = md.stations(m["r_trail"], m["chord_trail"], m["twist_trail"], m["nfoil_trail"])
    nt = ser["time"].size
    inp = dict(quarter=kin["quarter"], trail=kin["trail"], bound=kin["bound"], bxn=kin["bxn"],
               byn=kin["byn"], bzn=kin["bzn"], vblade=kin["vblade"], infty=ser["wind"],
               time=ser["time"], tsr=ser["tsr"], tip_rad=float(m["r_trail"][-1]), chord=st["chord"],
               nfoil=st["nfoil"], tables=m["tables"], cl0=cl0)
    user = dict(d=d, co=co, integ=integ, tol=tol, maxiter=maxiter, relax=relax, hz=ser["_hz"])
    loads = dict(twist_deg=st["twist"] + ser["_pitch"], r=st["r_nodes"], dr=st["dr"],
                 rpm=np.full(nt, ser["_omega"] * 30.0 / np.pi), rho=rho)
    return winds_ref.WInDSRun(inp, user, loads=loads)
