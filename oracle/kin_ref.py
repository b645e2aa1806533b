"""FP64 oracle of the blade kinematics (test infrastructure).

Restates, for a rotor (not the elliptical-wing platform type):
  * ``core/DCMRot.m:27-75`` -- direction cosine matrix of a rotation
    sequence: ``A <- R_k A`` for every rotation in order, ``y = A x``, with
    ``Rx = [1 0 0; 0 c -s; 0 s c]``, ``Ry = [c 0 s; 0 1 0; -s 0 c]``,
    ``Rz = [c -s 0; s c 0; 0 0 1]`` and ``c, s = cosd, sind`` of the angle;
  * ``core/kinematics.m`` -- hub position (platform motion plus the nominal
    hub rotated by ``[PtfmYaw PtfmPitch PtfmRoll NacYaw]``, sequence 'zyxz'),
    blade points (lead, bound, collocation, quarter chord, trailing edge,
    end) through the sequence 'zzzyxxyzxyz' of
    ``[twist, 90, pitch, precone, Az_b, Azimuth, ShftTilt, NacYaw, PtfmRoll,
    PtfmPitch, PtfmYaw]`` plus the hub;
  * ``core/velocity.m:36-88`` -- bound-point velocity by ``ctdiff`` over time,
    ``vel.bound = -d(pos.bound)/dt + wind``, the blade frames
    ``bxn = unit(end - bound)``, ``bzn = unit(diff(bound))`` (first row
    repeated), ``byn = bzn x bxn`` (and ``bxt, bzt, byt`` from the quarter-chord
    and trailing-edge nodes), ``vel.blade = [bxn; byn; bzn] . vel.bound``;
  * ``numerical/ctdiff.m`` -- O(h^2) one-sided ends, O(h^2) centred second and
    second-to-last, O(h^4) centred interior, ``dx = |mean(diff(t))|``.

``sind``/``cosd`` reduce the angle by the nearest multiple of 90 degrees
first, so multiples of 90 give exact 0 and +-1 as MATLAB's functions do.
Arrays use WInDS's layout [node, xyz, step, blade].
"""
from __future__ import annotations

import numpy as np

SEQ_ROTOR = "zzzyxxyzxyz"
SEQ_HUB = "zyxz"


def sincosd(t):
    """(sind(t), cosd(t)) with the argument reduced by the nearest multiple of
    90 degrees before conversion to radians."""
    t = np.asarray(t, dtype=np.float64)
    n = np.round(t / 90.0)
    r = np.radians(t - 90.0 * n)
    s0, c0 = np.sin(r), np.cos(r)
    q = np.mod(n, 4).astype(int)
    s = np.choose(q, [s0, c0, -s0, -c0])
    c = np.choose(q, [c0, -s0, -c0, s0])
    return s, c


def rot(axis, t):
    """Rotation matrices [..., 3, 3] of DCMRot for angle(s) t in degrees."""
    s, c = sincosd(t)
    o, z = np.ones_like(s), np.zeros_like(s)
    if axis == "x":
        rows = [[o, z, z], [z, c, -s], [z, s, c]]
    elif axis == "y":
        rows = [[c, z, s], [z, o, z], [-s, z, c]]
    else:
        rows = [[c, -s, z], [s, c, z], [z, z, o]]
    return np.stack([np.stack(r, -1) for r in rows], -2)


def dcm(angles, seq):
    """angles [..., len(seq)] (deg) -> A [..., 3, 3]: A <- R_k A in order,
    each product summed left to right as DCMRot's sum(R.*A, 2)."""
    angles = np.asarray(angles, dtype=np.float64)
    A = np.broadcast_to(np.eye(3), angles.shape[:-1] + (3, 3)).copy()
    for k, ax in enumerate(seq):
        R = rot(ax, angles[..., k])
        B = np.empty_like(A)
        for i in range(3):
            for j in range(3):
                B[..., i, j] = (R[..., i, 0] * A[..., 0, j] + R[..., i, 1] * A[..., 1, j]) + R[..., i, 2] * A[..., 2, j]
        A = B
    return A


def apply(A, x):
    """y = A x, each component summed left to right."""
    return np.stack([(A[..., i, 0] * x[..., 0] + A[..., i, 1] * x[..., 1]) + A[..., i, 2] * x[..., 2]
                     for i in range(3)], -1)


def ctdiff(t, y, axis):
    """numerical/ctdiff.m along ``axis`` (needs >= 5 samples)."""
    dx = abs(np.mean(np.diff(t)))
    y = np.moveaxis(np.asarray(y, dtype=np.float64), axis, 0)
    d = np.zeros_like(y)
    d[0] = (-y[2] + 4 * y[1] - 3 * y[0]) / (2 * dx)
    d[1] = (y[2] - y[0]) / (2 * dx)
    d[2:-2] = (-y[4:] + 8 * y[3:-1] - 8 * y[1:-3] + y[:-4]) / (12 * dx)
    d[-2] = (y[-1] - y[-3]) / (2 * dx)
    d[-1] = (3 * y[-1] - 4 * y[-2] + y[-3]) / (2 * dx)
    return np.moveaxis(d, 0, axis)


def unit(v, axis=1):
    return v / np.sqrt((v ** 2).sum(axis, keepdims=True))


def kinematics(r):
    """``r``: dict with time[nt], azimuth[nt], pitch[nt, nb], nac_yaw[nt],
    ptfm[nt, 6] (surge, sway, heave, roll, pitch, yaw), wind[nt, 3],
    r_trail/chord_trail/twist_trail[nst], r_nodes/chord/twist[ns] (deg),
    overhang, shaft_tilt, tower_ht, twr2shft, ptfm_ref, precone[nb].
    Returns the position, frame and velocity arrays of kinematics.m and
    velocity.m."""
    nt, nb = len(r["time"]), len(r["precone"])
    pf = np.asarray(r["ptfm"], np.float64)
    tilt = r["shaft_tilt"]
    hub_nom = np.array([r["overhang"] * sincosd(tilt)[1], 0.0,
                        r["ptfm_ref"] + r["tower_ht"] + r["twr2shft"] + r["overhang"] * sincosd(tilt)[0]])
    hub_seq = np.stack([pf[:, 5], pf[:, 4], pf[:, 3], r["nac_yaw"]], -1)       # [nt, 4]
    hub = pf[:, :3] + apply(dcm(hub_seq, SEQ_HUB), np.broadcast_to(hub_nom, (nt, 3)))
    az_b = 360.0 / nb * np.arange(nb)
    rt, ct, tt = (np.asarray(r[k], np.float64) for k in ("r_trail", "chord_trail", "twist_trail"))
    rn, cn, tn = (np.asarray(r[k], np.float64) for k in ("r_nodes", "chord", "twist"))
    zt, zn = np.zeros_like(rt), np.zeros_like(rn)
    local = {"lead": (np.stack([-0.25 * ct, zt, rt], -1), tt), "quarter": (np.stack([zt, zt, rt], -1), tt),
             "trail": (np.stack([0.75 * ct, zt, rt], -1), tt), "bound": (np.stack([zn, zn, rn], -1), tn),
             "colloc": (np.stack([0.25 * cn, zn, rn], -1), tn), "end": (np.stack([0.75 * cn, zn, rn], -1), tn)}
    out = {"hub": hub}
    for name, (pts, tw) in local.items():
        npt = pts.shape[0]
        res = np.zeros((npt, 3, nt, nb))
        for b in range(nb):
            ang = np.zeros((npt, nt, 11))
            ang[..., 0] = tw[:, None]
            ang[..., 1] = 90.0
            ang[..., 2] = np.asarray(r["pitch"])[None, :, b]
            ang[..., 3] = r["precone"][b]
            ang[..., 4] = az_b[b]
            ang[..., 5] = np.asarray(r["azimuth"])[None, :]
            ang[..., 6] = tilt
            ang[..., 7] = np.asarray(r["nac_yaw"])[None, :]
            ang[..., 8] = pf[None, :, 3]
            ang[..., 9] = pf[None, :, 4]
            ang[..., 10] = pf[None, :, 5]
            y = apply(dcm(ang, SEQ_ROTOR), np.broadcast_to(pts[:, None, :], (npt, nt, 3)))
            res[:, :, :, b] = np.moveaxis(y + hub[None, :, :], -1, 1)
        out[name] = res
    # velocity.m
    vb = -ctdiff(r["time"], out["bound"], axis=2) + np.asarray(r["wind"], np.float64).T[None, :, :, None]
    bxt = unit(out["trail"] - out["quarter"])
    bzt = unit(np.diff(out["quarter"], axis=0))
    bzt = np.concatenate([bzt[:1], bzt], axis=0)
    byt = np.cross(bzt, bxt, axis=1)
    bxn = unit(out["end"] - out["bound"])
    bzn = unit(np.diff(out["bound"], axis=0))
    bzn = np.concatenate([bzn[:1], bzn], axis=0)
    byn = np.cross(bzn, bxn, axis=1)
    vblade = np.stack([(f * vb).sum(1) for f in (bxn, byn, bzn)], axis=1)
    out.update(vbound=vb, bxn=bxn, byn=byn, bzn=bzn, bxt=bxt, byt=byt, bzt=bzt, vblade=vblade)
    return out
