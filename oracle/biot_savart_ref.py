"""FP64 CPU oracle for the WInDS induced-velocity path (test infrastructure).

This module is the checker, never the product: only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference legs
import it. It restates the reference's MATLAB sources in NumPy, keeping their
loop order, operation order and special cases:

* ``biot_savart``      -- ``core/BiotSavart.m:36-119``
* ``filament_length``  -- ``core/FilamentLength.m:27-44``
* ``vcore_ref``        -- ``core/vcore.m:30-40`` (absolute-time growth)
* ``filamentmod_ref``  -- ``core/filamentmod.m:23-41`` (double sqrt kept)
* ``bookkeeping``      -- ``WInDS.m:131-140`` / ``numerical/pcc.m:43-49``
* ``fe`` / ``ab2`` / ``ab4`` / ``pcc_correct`` -- ``numerical/*.m``

Parity pinning: the reference ships no golden vectors for this path (its
``tests/*.m`` need ``.mat`` files that are not in the repository). The cut-off
branch is pinned against the reference's own compiled host loop
(``cuda/source/BiotSavartMex.cu:236-282``, built by ``oracle/Makefile`` into
``oracle/_ref``); the Vatistas branch is pinned by analytic known answers
(straight segment, polygon ring centre, core limits) in ``tests/``.
"""
from __future__ import annotations

import math

import numpy as np


def _pad4(shape):
    sp = list(shape)
    while len(sp) < 4:
        sp.append(1)
    return tuple(sp)


def visc_index(d):
    """``n`` from ``d``: ``str2double(d(5:end))`` when ``d`` contains 'visc',
    else 0 (``core/BiotSavart.m:49-53``). ``'visc'`` alone gives NaN."""
    if isinstance(d, str) and "visc" in d:
        s = d[4:]
        try:
            return float(s) if s.strip() else float("nan")
        except ValueError:
            return float("nan")
    return 0.0


def biot_savart(F1, F2, P, gamma, rc, d, co, type_):
    """``[uind, L] = BiotSavart(F1,F2,P,gamma,rc,d,co,type)``.

    Loops over targets ``k, j, i`` exactly as ``core/BiotSavart.m:80-116``
    and vectorises over every filament, like MATLAB does."""
    P = np.asarray(P, dtype=np.float64)
    sp = _pad4(P.shape)
    ns, nt, nb = sp[0], sp[2], sp[3]
    P4 = P.reshape(sp, order="F")
    uind = np.zeros(sp, order="F")
    n = visc_index(d)
    F1 = np.asarray(F1, dtype=np.float64)
    F2 = np.asarray(F2, dtype=np.float64)
    fs = _pad4(F1.shape)
    F1 = F1.reshape(fs, order="F")
    F2 = F2.reshape(fs, order="F")
    gamma = np.asarray(gamma, dtype=np.float64).reshape((fs[0], 1, fs[2], fs[3]), order="F")
    rc = np.asarray(rc, dtype=np.float64).reshape((fs[0], 1, fs[2], fs[3]), order="F")
    x1, y1, z1 = F1[:, 0:1], F1[:, 1:2], F1[:, 2:3]
    x2, y2, z2 = F2[:, 0:1], F2[:, 1:2], F2[:, 2:3]
    x2x1 = x2 - x1
    y2y1 = y2 - y1
    z2z1 = z2 - z1
    L = x2x1 ** 2 + y2y1 ** 2 + z2z1 ** 2
    if type_ == "length":
        return np.zeros(P.shape), np.sqrt(L)
    if type_ != "full":
        return uind, L
    dnum = 0.0 if n != 0 else float(d)
    g4pi_den = 4 * math.pi
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        for k in range(nb):
            for j in range(nt):
                for i in range(ns):
                    px, py, pz = P4[i, 0, j, k], P4[i, 1, j, k], P4[i, 2, j, k]
                    pxx1 = px - x1
                    pyy1 = py - y1
                    pzz1 = pz - z1
                    pxx2 = px - x2
                    pyy2 = py - y2
                    pzz2 = pz - z2
                    r1 = np.sqrt(pxx1 ** 2 + pyy1 ** 2 + pzz1 ** 2)
                    r2 = np.sqrt(pxx2 ** 2 + pyy2 ** 2 + pzz2 ** 2)
                    r1dr2 = pxx1 * pxx2 + pyy1 * pyy2 + pzz1 * pzz2
                    r1tr2 = r1 * r2
                    if n != 0:
                        Ldr12 = (x2x1 * pxx1 + y2y1 * pyy1 + z2z1 * pzz1) ** 2
                        Cnu = (r1 ** 2) - (Ldr12 / L)
                        Cnu = Cnu * (rc ** n + Cnu ** n) ** (-1.0 / n)
                        ubar = Cnu * gamma / g4pi_den * (r1 + r2) / (r1tr2 * (r1tr2 + r1dr2))
                    else:
                        ubar = (gamma / g4pi_den) * (r1 + r2) / (r1tr2 * (r1tr2 + r1dr2) + (dnum * L))
                    ubar[np.isnan(ubar) | np.isinf(ubar) | ((r1 > co) & (r2 > co))] = 0.0
                    for c, cross in enumerate((pyy1 * pzz2 - pzz1 * pyy2,
                                               pzz1 * pxx2 - pxx1 * pzz2,
                                               pxx1 * pyy2 - pyy1 * pxx2)):
                        t = ubar * cross
                        uind[i, c, j, k] = t.sum(axis=0).sum(axis=1).sum(axis=1)[0]
    return uind, L


def biot_savart_flat(x1, x2, gamma, rc, pts, d, co, chunk=64):
    """Same arithmetic as :func:`biot_savart` for flat filament lists
    ``x1, x2 [nf,3]`` and targets ``pts [np,3]``; vectorised over chunks of
    targets for speed. Returns ``[np, 3]``."""
    n = visc_index(d)
    dnum = 0.0 if n != 0 else float(d)
    x2x1 = x2 - x1
    L = np.sum(x2x1 * x2x1, axis=1)
    out = np.zeros((pts.shape[0], 3))
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        for s in range(0, pts.shape[0], chunk):
            p = pts[s:s + chunk, None, :]
            a = p - x1[None]
            b = p - x2[None]
            r1 = np.sqrt(a[..., 0] ** 2 + a[..., 1] ** 2 + a[..., 2] ** 2)
            r2 = np.sqrt(b[..., 0] ** 2 + b[..., 1] ** 2 + b[..., 2] ** 2)
            r1dr2 = a[..., 0] * b[..., 0] + a[..., 1] * b[..., 1] + a[..., 2] * b[..., 2]
            r1tr2 = r1 * r2
            if n != 0:
                Ldr12 = (x2x1[None, :, 0] * a[..., 0] + x2x1[None, :, 1] * a[..., 1]
                         + x2x1[None, :, 2] * a[..., 2]) ** 2
                Cnu = r1 ** 2 - Ldr12 / L[None]
                Cnu = Cnu * (rc[None] ** n + Cnu ** n) ** (-1.0 / n)
                ubar = Cnu * gamma[None] / (4 * math.pi) * (r1 + r2) / (r1tr2 * (r1tr2 + r1dr2))
            else:
                ubar = (gamma[None] / (4 * math.pi)) * (r1 + r2) / (r1tr2 * (r1tr2 + r1dr2) + dnum * L[None])
            ubar[np.isnan(ubar) | np.isinf(ubar) | ((r1 > co) & (r2 > co))] = 0.0
            cx = a[..., 1] * b[..., 2] - a[..., 2] * b[..., 1]
            cy = a[..., 2] * b[..., 0] - a[..., 0] * b[..., 2]
            cz = a[..., 0] * b[..., 1] - a[..., 1] * b[..., 0]
            out[s:s + chunk, 0] = np.sum(ubar * cx, axis=1)
            out[s:s + chunk, 1] = np.sum(ubar * cy, axis=1)
            out[s:s + chunk, 2] = np.sum(ubar * cz, axis=1)
    return out


def filament_length(F1, F2):
    """``core/FilamentLength.m:27-44``: ``sqrt(|F2-F1|^2)`` per filament."""
    dx = F2[:, 0:1] - F1[:, 0:1]
    dy = F2[:, 1:2] - F1[:, 1:2]
    dz = F2[:, 2:3] - F1[:, 2:3]
    return np.sqrt(dx ** 2 + dy ** 2 + dz ** 2)


def vcore_ref(gamma, r0, alpha, nu, a1, time_s):
    """``core/vcore.m:30-37``: ``rc = r0^2 + 4 alpha nu (1 + a1 |gamma|/nu) t``
    with the absolute simulation time ``t`` (squared radius)."""
    Re = np.abs(gamma / nu)
    return r0 ** 2 + 4 * alpha * nu * (1 + a1 * Re) * time_s


def vcore_age(gamma, rc0, alpha, nu, a1, delta, age_s):
    """Age-based growth used by the synthetic wakes:
    ``rc^2 = rc0^2 + 4 alpha delta nu age`` (``a1`` term kept as in vcore)."""
    Re = np.abs(gamma / nu)
    return rc0 ** 2 + 4 * alpha * delta * nu * (1 + a1 * Re) * age_s


def filamentmod_ref(rc_new, len_new, len_old):
    """``core/filamentmod.m:23-41`` on one filament family: interior columns
    ``2:end-1`` of the new lengths against columns ``2:end`` of the previous
    step; lengths are square-rooted again (the reference passes ``|L|``)."""
    out = rc_new.copy()
    new = np.sqrt(len_new[:, :, 1:-1])
    old = np.sqrt(len_old[:, :, 1:])
    strain = (new - old) / old
    out[:, :, 1:-1] = rc_new[:, :, 1:-1] * (1.0 / (1.0 + strain))
    return out


def bookkeeping(bound_new, trail_prev):
    """``WInDS.m:131-140``: new bound column -> trailing columns -> shed
    columns. ``bound_new [ns,1,1,nb]``, ``trail_prev [nst,1,m,nb]``.
    Returns ``(shed [ns,1,m+2,nb], trail [nst,1,m+1,nb])``."""
    ns, nb = bound_new.shape[0], bound_new.shape[3]
    z = np.zeros((1, 1, 1, nb))
    t0 = np.diff(np.concatenate([z, bound_new, z], axis=0), axis=0)
    trail = np.concatenate([t0, trail_prev], axis=2)
    c = np.cumsum(trail[:-1], axis=0)
    shed_rest = np.diff(np.concatenate([c, np.zeros((ns, 1, 1, nb))], axis=2), axis=2)
    shed = np.concatenate([bound_new, shed_rest], axis=2)
    return shed, trail


def fe(dom_t, vel_t, dt):
    """``numerical/fe.m:31``: columns 3:end of the new domain."""
    return dom_t[:, :, 1:] + dt * vel_t[:, :, 1:]


def ab2(dom_t, vel_t, vel_tm1, dt):
    """``numerical/ab2.m:38-39``."""
    nst, nb = dom_t.shape[0], dom_t.shape[3]
    prev = np.concatenate([np.zeros((nst, 3, 1, nb)), vel_tm1[:, :, 1:]], axis=2)
    return dom_t[:, :, 1:] + dt / 2 * (3 * vel_t[:, :, 1:] - prev)


def ab4(dom_t, vels, dt):
    """``numerical/ab4.m:77-81``; ``vels = [v_t, v_t-1, v_t-2, v_t-3]``."""
    nst, nb = dom_t.shape[0], dom_t.shape[3]
    z = lambda k: np.zeros((nst, 3, k, nb))
    v0, v1, v2, v3 = vels
    return dom_t[:, :, 1:] + dt / 24 * (
        55 * v0[:, :, 1:]
        - 59 * np.concatenate([z(1), v1[:, :, 1:]], axis=2)
        + 37 * np.concatenate([z(2), v2[:, :, 1:]], axis=2)
        - 9 * np.concatenate([z(3), v3[:, :, 1:]], axis=2))


def pcc_correct(dom_t, vel_t, vel_tp1, dt):
    """``numerical/pcc.m:74-75``: trapezoid corrector for columns 3:end."""
    return dom_t[:, :, 1:] + dt / 2 * (vel_tp1[:, :, 2:] + vel_t[:, :, 1:])
