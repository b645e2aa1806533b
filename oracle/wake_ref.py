"""FP64 oracle of the free-wake time step (test infrastructure).

Restates, for a wake kept at a fixed number of age columns ``na`` (the
oldest column is dropped each step, as the truncated-wake configurations do):

* Γ bookkeeping     -- ``WInDS.m:131-140`` / ``numerical/pcc.m:43-49``
* core growth       -- ``core/vcore.m:30-40`` (absolute time, ``core_mode=0``)
                       or the age form ``rc^2 = rc0^2 + 4 alpha delta nu (1+a1 Re) age``
                       (``core_mode=1``)
* lengths/stretch   -- ``core/FilamentLength.m:27-44``, ``core/filamentmod.m:23-41``:
                       new columns ``2:end-1`` against the previous step's columns of the
                       same index (the reference aligns by index), lengths square-rooted
                       again (the reference stores ``|L|`` and takes ``sqrt`` once more)
* induced velocity  -- ``core/BiotSavart.m`` (via the C oracle), shed + trailing
* convection        -- ``numerical/fe.m:31``, ``ab2.m:38-39``, ``ab4.m:77-81``,
                       ``pcc.m:37-75``; with ``pcc_double_add`` the corrector's induced
                       velocity is added to the next step's velocity as well, as
                       ``pcc.m:71`` followed by ``WInDS.m:168`` do

Column 0 and 1 of the domain are the quarter-chord and trailing-edge nodes from
the kinematics (``core/initials.m:85-86``); columns ``2:end`` are convected.
Arrays use WInDS's layout ``[span, xyz, age, blade]`` (Fortran-ordered).
"""
from __future__ import annotations

import dataclasses

import numpy as np

import oracle as orc


@dataclasses.dataclass
class WakeCaseRef:
    nst: int
    nb: int
    na: int
    dt: float
    t0: float
    quarter: np.ndarray    # [nst,3,nsteps,nb]
    trailing: np.ndarray   # [nst,3,nsteps,nb]
    wind: np.ndarray       # [3, nsteps]
    shear: float
    hub_height: float
    core_mode: int
    r0: float
    rc0: float
    alpha: float
    nu: float
    a1: float
    delta: float
    dom: np.ndarray        # [nst,3,na,nb]
    bound: np.ndarray      # [ns,nb]
    trail_gamma: np.ndarray  # [nst,na-1,nb]


def wind_at(case, s, pts):
    """Freestream at points ``pts [..., 3]`` for step ``s``: the step's wind
    vector scaled by ``((H + z) / H) ** shear`` (uniform when shear = 0)."""
    w = case.wind[:, s]
    if case.shear == 0.0:
        return np.broadcast_to(w, pts.shape).copy()
    h = np.maximum(case.hub_height + pts[..., 2], 1e-3) / case.hub_height
    return w * (h ** case.shear)[..., None]


def bookkeeping(bound, trail_prev):
    """Trailing and shed Γ from the bound column and the previous trailing
    columns (the oldest dropped): ``trail = [diff([0;G;0]), trail_prev(:,1:end-1)]``,
    ``shed = [G, diff(cat(cumsum(trail(1:end-1)), 0))]``."""
    nst, m, nb = trail_prev.shape
    ns = nst - 1
    z = np.zeros((1, nb))
    t0 = np.diff(np.concatenate([z, bound, z], axis=0), axis=0)       # [nst, nb]
    trail = np.concatenate([t0[:, None, :], trail_prev[:, : m - 1, :]], axis=1)
    c = np.cumsum(trail[:-1], axis=0)                                   # [ns, m, nb]
    rest = np.diff(np.concatenate([c, np.zeros((ns, 1, nb))], axis=1), axis=1)
    shed = np.concatenate([bound[:, None, :], rest], axis=1)            # [ns, m+1, nb]
    return shed, trail


def core(case, gamma, age_or_time):
    Re = np.abs(gamma / case.nu)
    if case.core_mode == 0:
        return case.r0 ** 2 + 4 * case.alpha * case.nu * (1 + case.a1 * Re) * age_or_time
    return case.rc0 ** 2 + 4 * case.alpha * case.delta * case.nu * (1 + case.a1 * Re) * age_or_time


def lengths(dom):
    sh = np.sqrt(np.sum((dom[1:] - dom[:-1]) ** 2, axis=1))                 # [ns, na, nb]
    tr = np.sqrt(np.sum((dom[:, :, :-1] - dom[:, :, 1:]) ** 2, axis=1))     # [nst, na-1, nb]
    return sh, tr


def cores(case, shed, trail, time, len_new, len_old, stretch):
    """``rc_eff`` for shed and trailing filaments (vcore + filamentmod)."""
    na = shed.shape[1]
    if case.core_mode == 0:
        ts, tt = time, time
    else:
        ts = np.arange(na)[None, :, None] * case.dt
        tt = (np.arange(na - 1)[None, :, None] + 0.5) * case.dt
    rcs = core(case, shed, ts)
    rct = core(case, trail, tt)
    if stretch and len_old is not None:
        sn, tn = len_new
        so, to = len_old
        for rc, new, old in ((rcs, sn, so), (rct, tn, to)):
            m = new.shape[1]
            a = np.sqrt(new[:, 1:m - 1])
            b = np.sqrt(old[:, 1:m - 1])
            strain = (a - b) / b
            rc[:, 1:m - 1] = rc[:, 1:m - 1] * (1.0 / (1.0 + strain))
    return rcs, rct


def induced(dom, shed, trail, rcs, rct, d, co):
    F1s, F2s = dom[:-1], dom[1:]
    F1t, F2t = dom[:, :, 1:], dom[:, :, :-1]
    u = orc.c_eval(F1s, F2s, dom, shed[:, None], rcs[:, None], d, co)
    u = u + orc.c_eval(F1t, F2t, dom, trail[:, None], rct[:, None], d, co)
    return u


class WakeRef:
    """One case's state and its step (the device engine's reference)."""

    def __init__(self, case: WakeCaseRef, integrator="pcc", d="visc2", co=1000.0,
                 pcc_double_add=True, stretch=True):
        self.c = case
        self.integ = integrator
        self.d, self.co = d, co
        self.double_add = pcc_double_add
        self.stretch = stretch
        self.step_idx = 0
        self.dom = case.dom.copy(order="F")
        self.bound = case.bound.copy()
        # trailing columns of the step before (trail_prev(:, k) = trail(:, k+1)); each
        # step forms its Γ from them and the bound column (WInDS.m:131-140)
        self.trail_prev = np.zeros_like(case.trail_gamma)
        self.trail_prev[:, :-1] = case.trail_gamma[:, 1:]
        self.len_old = None
        self.vel_hist = []        # previous velocities, newest first
        self.vel_carry = None     # pcc: induced velocity carried into the next step

    def time(self, s):
        return self.c.t0 + s * self.c.dt

    def _eval(self, dom, shed, trail, time, len_old):
        ln = lengths(dom)
        rcs, rct = cores(self.c, shed, trail, time, ln, len_old, self.stretch)
        return induced(dom, shed, trail, rcs, rct, self.d, self.co), ln, rcs, rct

    def _nodes(self, dom):
        return np.moveaxis(dom, 1, -1)  # [nst, na, nb, 3]

    def _wind(self, s, dom):
        w = wind_at(self.c, s, self._nodes(dom))
        return np.moveaxis(w, -1, 1)

    def _before_commit(self, s):
        """Runs after the convection of step ``s``, with the step's positions,
        Γ and cores still current (the Kutta-Joukowski solve: WInDS.m:182)."""

    def step(self):
        """One time step p -> p+1; returns the induced velocity at p."""
        c, s = self.c, self.step_idx
        self.shed, self.trail = bookkeeping(self.bound, self.trail_prev)
        u, ln, self.rcs, self.rct = self._eval(self.dom, self.shed, self.trail, self.time(s), self.len_old)
        vel = self._wind(s, self.dom) + u
        if self.vel_carry is not None:
            vel = vel + self.vel_carry
        self.len_old = ln
        self.uind = u
        new = np.empty_like(self.dom)
        new[:, :, 0] = c.quarter[:, :, s + 1]
        new[:, :, 1] = c.trailing[:, :, s + 1]
        tail = self.dom[:, :, 1:-1]
        if self.integ == "fe":
            new[:, :, 2:] = tail + c.dt * vel[:, :, 1:-1]
        elif self.integ == "ab2":
            if not self.vel_hist:  # no previous velocity yet: forward Euler (ab2.m:35-36)
                new[:, :, 2:] = tail + c.dt * vel[:, :, 1:-1]
            else:
                sh = np.zeros_like(vel[:, :, 1:-1])
                sh[:, :, 1:] = self.vel_hist[0][:, :, 1:-2]
                new[:, :, 2:] = tail + c.dt / 2 * (3 * vel[:, :, 1:-1] - sh)
        elif self.integ == "ab4":
            def shifted(k):
                out = np.zeros_like(vel[:, :, 1:-1])
                if len(self.vel_hist) >= k:
                    out[:, :, k:] = self.vel_hist[k - 1][:, :, 1:-1 - k]
                return out
            if len(self.vel_hist) < 3:  # forward Euler until three past velocities exist
                new[:, :, 2:] = tail + c.dt * vel[:, :, 1:-1]
            else:
                new[:, :, 2:] = tail + c.dt / 24 * (55 * vel[:, :, 1:-1] - 59 * shifted(1)
                                                    + 37 * shifted(2) - 9 * shifted(3))
        elif self.integ == "pcc":
            new[:, :, 2:] = tail + c.dt * vel[:, :, 1:-1]            # fe predictor
            shed1, trail1 = bookkeeping(self.bound, self.trail)
            u1, _, _, _ = self._eval(new, shed1, trail1, self.time(s + 1), ln)
            vel1 = self._wind(s + 1, new) + u1
            new[:, :, 2:] = tail + c.dt / 2 * (vel1[:, :, 2:] + vel[:, :, 1:-1])
            self.vel_carry = u1 if self.double_add else None
        else:
            raise ValueError(self.integ)
        self.vel_hist = [vel] + self.vel_hist[:2]
        self._before_commit(s)
        self.dom = np.asfortranarray(new)
        self.trail_prev = self.trail
        self.step_idx += 1
        return u
