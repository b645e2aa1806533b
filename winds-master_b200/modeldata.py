"""Rotor model inputs in WInDS's own formats, and the wake / lifting-line
cases built from them through the kinematics.

  * ``read_airfoil(path)`` -- an AeroDyn airfoil table as
    ``modeldata/NRELrotor.m:131-133`` reads it: 14 header lines, then rows of
    AoA (deg), Cl, Cd, Cm; of two rows with the same AoA the first is dropped.
  * ``stations(...)`` -- the blade stations of ``NRELrotor.m:40-47``: midpoints
    of the trailing nodes, chord and twist interpolated linearly, the airfoil
    index of the nearest trailing node (ties to the outer node), widths.
  * ``operating_series(...)`` -- the turbine time series of ``NRELrotor.m``
    for a constant wind, tip-speed ratio, pitch and nacelle yaw with the
    platform at rest (``fastout.Azimuth = omega t``, ``RotSpeed``), from
    ``t = -(na - 1) dt`` so the initial wake has a history.
  * ``read_fast_out(path, t)`` -- a FAST output file as
    ``core/output_import.m:37-72`` reads it: channel names on line 7, units
    on line 8, tab-separated samples after; every channel interpolated
    linearly to ``t0 : 1/freq : t1`` (clamped to the recorded times).
  * ``series_from_fastout(model, fo)`` -- the kinematics inputs of a FAST time
    series (``fastout.Azimuth``, ``BldPitch1..nb``, ``NacYaw``, ``Ptfm*``,
    ``WindV*i``, ``RotSpeed``), in the form ``operating_series`` returns.
  * ``cases(...)`` -- a ``winds_wake_case`` and a ``winds_kj_case`` (dicts for
    ``wake.WakeBatch`` / ``set_kj``) from the kinematics of that series.
  * ``initial_cases(...)`` -- the same for a run from ``core/initials.m``'s
    state: a wake of two columns that grows by one per step, the core of
    ``core/vcore.m`` with ``wake.r0`` and ``fastout.Time`` per step.
"""
from __future__ import annotations

import numpy as np

RHO = 1.225


def read_airfoil(path: str) -> dict:
    rows = []
    with open(path) as f:
        lines = f.read().splitlines()
    for line in lines[14:]:
        parts = line.split()
        if len(parts) < 4:
            continue
        try:
            rows.append([float(p) for p in parts[:4]])
        except ValueError:
            break
    a = np.asarray(rows, dtype=np.float64)
    keep = np.ones(len(a), dtype=bool)
    keep[:-1] = np.diff(a[:, 0]) != 0  # NRELrotor.m:132-133
    a = a[keep]
    return dict(aoa=a[:, 0], cl=a[:, 1], cd=a[:, 2], cm=a[:, 3])


def stations(r_trail, chord_trail, twist_trail, nfoil_trail) -> dict:
    """Blade stations from trailing-node data (NRELrotor.m:40-47); ``nfoil``
    is returned 1-based as in WInDS."""
    rt = np.asarray(r_trail, np.float64)
    rn = rt[:-1] + np.diff(rt) / 2
    idx = np.searchsorted(rt, rn)               # rt[idx-1] < rn <= rt[idx]
    lo = rt[idx - 1]
    hi = rt[np.minimum(idx, len(rt) - 1)]
    nearest = np.where(rn - lo < hi - rn, idx - 1, idx)
    return dict(r_nodes=rn, chord=np.interp(rn, rt, chord_trail), twist=np.interp(rn, rt, twist_trail),
                nfoil=np.asarray(nfoil_trail)[nearest].astype(np.int64), dr=np.abs(np.diff(rt)))


def operating_series(model: dict, U=11.4, tsr=7.0, pitch=0.0, yaw=0.0, hz=10.0, nsteps=51,
                     na=40) -> dict:
    """Turbine time series (kinematics inputs) of a steady operating point,
    samples ``-(na-1) .. nsteps`` at ``hz``."""
    R = float(model["r_trail"][-1])
    omega = tsr * U / R
    t = (np.arange(-(na - 1), nsteps + 1)) / hz
    nt, nb = t.size, int(model["nb"])
    st = stations(model["r_trail"], model["chord_trail"], model["twist_trail"], model["nfoil_trail"])
    wind = np.zeros((nt, 3))
    wind[:, 0] = U
    return dict(time=t, azimuth=omega * (180.0 / np.pi) * t, pitch=np.full((nt, nb), pitch),
                nac_yaw=np.full(nt, yaw), ptfm=np.zeros((nt, 6)), wind=wind,
                r_trail=model["r_trail"], chord_trail=model["chord_trail"],
                twist_trail=model["twist_trail"], r_nodes=st["r_nodes"], chord=st["chord"],
                twist=st["twist"], precone=np.full(nb, model["precone"]), overhang=model["overhang"],
                shaft_tilt=model["shaft_tilt"], tower_ht=model["tower_ht"], twr2shft=model["twr2shft"],
                ptfm_ref=0.0, _omega=omega, _U=U, _pitch=pitch, _na=na, _nsteps=nsteps, _hz=hz)


FAST_CHANNELS = ("Time", "Azimuth", "NacYaw", "PtfmSurge", "PtfmSway", "PtfmHeave", "PtfmRoll",
                 "PtfmPitch", "PtfmYaw", "WindVxi", "WindVyi", "WindVzi", "RotSpeed")


def read_fast_out(path: str, t=(-float("inf"), float("inf"), 0.0), dt=None, verbose=False) -> dict:
    """Channels of a FAST output file (output_import.m:37-72): line 7 holds the
    tab-separated channel names, line 8 the units, the samples follow.
    ``dt``, when given (the .fst integration step of a non-Simulink run,
    output_import.m:44-46), regrids the time column as ``t_first:dt:t_last``.
    ``t = (t0, t1, freq)``: every channel is interpolated linearly to
    ``t0 : 1/freq : t1``, with t0 and t1 clamped to the recorded range;
    ``freq == 0`` keeps the file's mean sample rate. (The reference takes that
    rate from differences along the first sample row, across channels; the
    time column is what it means.) Returns name -> array, plus ``units``."""
    with open(path) as f:
        lines = f.read().splitlines()
    names = lines[6].split("\t")
    names = [n.strip() for n in names if n.strip()]
    units = [u.strip() for u in lines[7].split("\t") if u.strip()]
    rows = [[float(v) for v in ln.split()] for ln in lines[8:] if ln.strip()]
    data = np.asarray(rows, dtype=np.float64)
    if data.ndim != 2 or data.shape[1] != len(names):
        raise ValueError(f"{path}: {len(names)} channel names, samples of width {data.shape}")
    if dt is not None:
        data[:, 0] = data[0, 0] + dt * np.arange(data.shape[0])
    t0, t1, freq = (float(x) for x in t)
    if freq == 0.0:
        freq = 1.0 / float(np.mean(np.diff(data[:, 0])))
    if t0 < data[0, 0]:
        t0 = float(data[0, 0])
        if verbose:
            print(f"User selected initial time out-of-range, reset to {t0:g} seconds.")
    if t1 > data[-1, 0]:
        t1 = float(data[-1, 0])
        if verbose:
            print(f"User selected final time out-of-range, reset to {t1:g} seconds.")
    n = int(np.floor((t1 - t0) * freq + 1e-9)) + 1
    ti = t0 + np.arange(n) / freq
    out = {"units": dict(zip(names, units))}
    out[names[0]] = ti
    for k, name in enumerate(names[1:], start=1):
        out[name] = np.interp(ti, data[:, 0], data[:, k])
    return out


def series_from_fastout(model: dict, fo: dict, na: int = 40) -> dict:
    """Kinematics inputs of a FAST time series (kinematics.m:27-109 reads
    these channels), in ``operating_series``'s form: the first ``na - 1``
    samples make the initial wake's history and step 0 is sample ``na - 1``.
    The blade pitch goes to the loads per step and blade (``pitch``), as
    perform.m:22-33 uses fastout.BldPitch<b>."""
    nb = int(model["nb"])
    t = np.asarray(fo["Time"], np.float64)
    nt = t.size
    if nt < na + 1:
        raise ValueError(f"{nt} samples; the initial wake needs na = {na} plus a step")
    pitch = np.stack([np.asarray(fo[f"BldPitch{b + 1}"], np.float64) for b in range(nb)], 1)
    ptfm = np.stack([np.asarray(fo[k], np.float64) for k in
                     ("PtfmSurge", "PtfmSway", "PtfmHeave", "PtfmRoll", "PtfmPitch", "PtfmYaw")], 1)
    wind = np.stack([np.asarray(fo[k], np.float64) for k in ("WindVxi", "WindVyi", "WindVzi")], 1)
    st = stations(model["r_trail"], model["chord_trail"], model["twist_trail"], model["nfoil_trail"])
    hz = 1.0 / float(np.mean(np.diff(t)))
    omega = float(np.mean(fo["RotSpeed"])) * np.pi / 30.0
    return dict(time=t, azimuth=np.asarray(fo["Azimuth"], np.float64), pitch=pitch,
                nac_yaw=np.asarray(fo["NacYaw"], np.float64), ptfm=ptfm, wind=wind,
                r_trail=model["r_trail"], chord_trail=model["chord_trail"],
                twist_trail=model["twist_trail"], r_nodes=st["r_nodes"], chord=st["chord"],
                twist=st["twist"], precone=np.full(nb, model["precone"]), overhang=model["overhang"],
                shaft_tilt=model["shaft_tilt"], tower_ht=model["tower_ht"], twr2shft=model["twr2shft"],
                ptfm_ref=0.0, rpm=np.asarray(fo["RotSpeed"], np.float64), _omega=omega,
                _U=float(np.mean(wind[:, 0])), _pitch=float(pitch.mean()), _na=na,
                _nsteps=nt - na, _hz=hz, _pitch_per_step=True)


def write_fast_out(path: str, channels: dict, title: str = "synthetic FAST output") -> None:
    """Writes ``channels`` (name -> array, ``Time`` first) in the layout
    ``read_fast_out`` reads: six header lines, names, units, samples."""
    names = list(channels)
    units = {"Time": "(s)", "Azimuth": "(deg)", "NacYaw": "(deg)", "RotSpeed": "(rpm)"}
    with open(path, "w") as f:
        f.write(f"{title}\n\n\n\n\n\n")
        f.write("\t".join(names) + "\n")
        f.write("\t".join(units.get(n, "(deg)" if "Pitch" in n or n[-3:] in ("oll", "Yaw")
                                     else "(m)" if n.startswith("Ptfm") else "(m/s)")
                          for n in names) + "\n")
        data = np.stack([np.asarray(channels[n], np.float64) for n in names], 1)
        for row in data:
            f.write("\t".join(f"{v:.10E}" for v in row) + "\n")


def cases(model: dict, series: dict, kin: dict, rc0=0.1, delta=100.0, nu=1.5e-5, alpha=1.25643) -> tuple:
    """(wake case, lifting-line case) from a series and its kinematics
    ``kin`` (device ``kin.kinematics`` or the oracle): step 0 at t = 0, the
    wake's older columns the trailing edge of earlier steps convected with the
    wind; bound circulation starting at zero."""
    na, nsteps, hz, U = series["_na"], series["_nsteps"], series["_hz"], series["_U"]
    s0 = na - 1
    nb = int(model["nb"])
    nst = len(model["r_trail"])
    ns = nst - 1
    dt = 1.0 / hz
    f = np.asfortranarray
    quarter = kin["quarter"][:, :, s0:, :]
    trail = kin["trail"][:, :, s0:, :]
    dom = np.zeros((nst, 3, max(na, 2), nb))  # initial_cases sets the capacity of na = 1 series
    dom[:, :, 0, :] = quarter[:, :, 0, :]
    dom[:, :, 1, :] = trail[:, :, 0, :]
    for j in range(2, na):
        te = kin["trail"][:, :, s0 - (j - 1), :].copy()
        te[:, 0, :] += U * (j - 1) * dt
        dom[:, :, j, :] = te
    wind = np.zeros((3, nsteps + 1))
    wind[0] = U
    wake = dict(nst=nst, nb=nb, na=na, nsteps=nsteps + 1, dt=dt, t0=0.0, quarter=f(quarter),
                trailing=f(trail), wind=f(wind), shear=0.0, hub_height=float(model["tower_ht"]),
                core_mode=1, r0=rc0, rc0=rc0, alpha=alpha, nu=nu, a1=0.0, delta=delta, dom=f(dom),
                bound=f(np.zeros((ns, nb))), trail_gamma=f(np.zeros((nst, max(na, 2) - 1, nb))))
    st = stations(model["r_trail"], model["chord_trail"], model["twist_trail"], model["nfoil_trail"])
    tabs = model["tables"]
    R = float(model["r_trail"][-1])
    az = np.radians(series["azimuth"][s0:])[:, None] + 2 * np.pi * np.arange(nb)[None, :] / nb
    per_step = bool(series.get("_pitch_per_step", False))
    kj = dict(ll=f(kin["bound"][:, :, s0:, :]), bxn=f(kin["bxn"][:, :, s0:, :]),
              byn=f(kin["byn"][:, :, s0:, :]), bzn=f(kin["bzn"][:, :, s0:, :]),
              vblade=f(kin["vblade"][:, :, s0:, :]), chord=st["chord"],
              foil=(st["nfoil"] - 1).astype(np.int32),
              foil_points=np.array([len(t["aoa"]) for t in tabs], dtype=np.int32),
              aoa=np.concatenate([t["aoa"] for t in tabs]), cl=np.concatenate([t["cl"] for t in tabs]),
              cd=np.concatenate([t["cd"] for t in tabs]), r_over_R=st["r_nodes"] / R,
              chord_over_R=st["chord"] / R,
              twist=np.radians(st["twist"] + (0.0 if per_step else series["_pitch"])),
              azimuth=f(az), r_station=st["r_nodes"], dr_station=st["dr"],
              rpm=(np.asarray(series["rpm"][s0:s0 + nsteps + 1], np.float64) if "rpm" in series
                   else np.full(nsteps + 1, series["_omega"] * 30.0 / np.pi)), rho=RHO)
    if per_step:  # blade pitch per step and blade for the loads (perform.m:22-33)
        kj["pitch"] = f(np.asarray(series["pitch"], np.float64)[s0:s0 + nsteps + 1])
    return wake, kj


VCORE = dict(alpha=1.25643, nu=1e-5, delta=100.0, a1=6.5e-5)  # core/constants.m:22-25


def initial_r0(tip_rad, tsr, wind_speed, alpha=VCORE["alpha"], nu=VCORE["nu"], delta=VCORE["delta"]):
    """``wake.r0`` per step (core/initials.m:134-135):
    ``sqrt(4 alpha nu delta T0)``, ``T0 = 2 pi R / (12 TSR |U|)``."""
    T0 = 2 * np.pi * tip_rad / (12 * np.asarray(tsr, np.float64) * np.asarray(wind_speed, np.float64))
    return np.sqrt(4 * alpha * nu * delta * T0)


def initial_cases(model: dict, series: dict, kin: dict, cl0, na: int, rho=1.23) -> tuple:
    """(wake case, lifting-line case) of a run from the state core/initials.m
    sets up at time index 1 (step 0 of the series, ``series["_na"] == 1``):
    ``wake.domain{1}`` = quarter-chord and trailing-edge nodes, capacity ``na``
    columns; bound circulation ``0.5 |U(1)| chord cl0`` (``cl0``: BEM's Cl,
    [ns] or [ns, nb]); ``tsr`` per step from ``series["tsr"]`` (else
    omega R / |U|) for ``wake.r0``; the core of core/vcore.m (absolute time,
    core/constants.m's values). Use with ``startup="reference"``."""
    if series["_na"] != 1:
        raise ValueError("a run from initials starts at the series' first sample (na = 1)")
    wk, kj = cases(model, series, kin)
    nst, nb, nsteps = wk["nst"], wk["nb"], wk["nsteps"]
    ns = nst - 1
    wind = np.asarray(series["wind"], np.float64)[:nsteps]
    U = np.sqrt(np.sum(wind ** 2, axis=1))
    R = float(model["r_trail"][-1])
    tsr = np.asarray(series["tsr"], np.float64)[:nsteps] if "tsr" in series else series["_omega"] * R / U
    dom = np.zeros((nst, 3, na, nb))
    dom[:, :, :2, :] = wk["dom"][:, :, :2, :]
    cl0 = np.asarray(cl0, np.float64)
    if cl0.ndim == 1:
        cl0 = np.repeat(cl0[:, None], nb, axis=1)
    chord = np.asarray(kj["chord"], np.float64)
    bound = 0.5 * U[0] * chord[:, None] * cl0
    wk.update(na=na, na_start=2, dom=np.asfortranarray(dom), bound=np.asfortranarray(bound),
              trail_gamma=np.asfortranarray(np.zeros((nst, na - 1, nb))), wind=np.asfortranarray(wind.T),
              core_mode=0, r0=0.0, time=np.asarray(series["time"], np.float64)[:nsteps].copy(),
              r0_step=initial_r0(R, tsr, U), **VCORE)
    kj["rho"] = rho
    return wk, kj


def load_model(path: str) -> dict:
    """A rotor model saved as by ``tests/golden/make_nrel.py``: trailing-node
    geometry, airfoil index, turbine constants and the airfoil tables."""
    d = np.load(path, allow_pickle=False)
    names = [str(n) for n in d["names"]]
    model = {k: d[k] for k in ("r_trail", "chord_trail", "twist_trail", "nfoil_trail")}
    for k in ("nb", "tower_ht", "twr2shft", "shaft_tilt", "precone", "overhang"):
        model[k] = float(d[k]) if k != "nb" else int(d[k])
    model["names"] = names
    model["tables"] = [dict(aoa=d[f"aoa_{k}"], cl=d[f"cl_{k}"], cd=d[f"cd_{k}"]) for k in range(len(names))]
    return model
