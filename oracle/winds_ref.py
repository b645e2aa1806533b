"""FP64 oracle of the WInDS driver's time loop, literally (test infrastructure).

Restates ``WInDS.m:127-182`` from the state ``core/initials.m:37-152`` sets
up, keeping the reference's growing cell arrays: at time index ``p`` (1-based,
as in MATLAB) ``wake.domain{p}`` has ``p+1`` age columns, ``gamma.shed{p}``
``p+1`` and ``gamma.trail{p}`` ``p`` columns. Per step:

* Γ bookkeeping             ``WInDS.m:131-140``
* core growth, stretching   ``core/vcore.m:30-51`` with ``wake.r0(time)`` and
                            ``fastout.Time(time)``; ``core/FilamentLength.m:27-44``;
                            ``core/filamentmod.m:23-41`` (``time>3``, double sqrt)
* induced velocity          ``BiotSavart(...,'full')`` of the shed and trailing
                            filaments at every node (``WInDS.m:157-168``), through
                            the C restatement of ``core/BiotSavart.m``
* convection                ``numerical/fe.m:31``, ``ab2.m:35-39``, ``ab4.m:35-42``,
                            ``pcc.m:37-75`` with their time-index switches and the
                            corrector's second addition of its induced velocity
                            (``pcc.m:71`` then ``WInDS.m:168``)
* Kutta-Joukowski           ``core/KuttaJoukowski.m:42-49`` (fixed point) and
                            ``kj()`` ``:173-298``
* loads                     ``postproc/perform.m:18-62`` per step (``perform_ref``)

Not restated: BEM (``core/initials.m:116``); its Cl at the first step is an
input (``cl0``), as is everything the kinematics compute (``pos``, ``vel.blade``).
Arrays keep WInDS's layout ``[span, xyz, age, blade]``; the singleton second
dimension of Γ, cores and lengths is dropped (``[span, age, blade]``).
"""
from __future__ import annotations

import math

import numpy as np

import oracle as orc
import perform_ref
from kj_ref import KJDiverged, interp1

CONST = dict(alpha=1.25643, nu=1e-5, delta=100.0, a1=6.5e-5, rho=1.23)  # core/constants.m:22-28


def _diff_span(G):
    """``diff([zeros(1,1,1,nb); G; zeros(1,1,1,nb)], 1)`` for ``G [ns, nb]``."""
    z = np.zeros((1, G.shape[1]))
    return np.diff(np.concatenate([z, G, z], axis=0), axis=0)


def _shed_rest(trail, ns):
    """``diff(cat(3, cumsum(trail(1:end-1,:,:,:), 1), zeros(ns,1,1,nb)), 1, 3)``."""
    c = np.cumsum(trail[:-1], axis=0)
    z = np.zeros((ns, 1, trail.shape[2]))
    return np.diff(np.concatenate([c, z], axis=1), axis=1)


class WInDSRun:
    """One rotor's run. Inputs (0-based time index ``k = p - 1``):

    ``quarter, trail [nst,3,nt,nb]`` (pos.quarter, pos.trail), ``bound,
    bxn, byn, bzn, vblade [ns,3,nt,nb]`` (pos.bound, pos.nodes.b?n,
    vel.blade), ``infty [nt,3]`` (wind.infty), ``time [nt]`` (fastout.Time),
    ``tsr [nt]`` (fastout.TipSpdRat), ``tip_rad`` (blade.TipRad), ``chord
    [ns]``, ``nfoil [ns]`` (1-based, blade.NFoil), ``tables`` (list of dicts
    aoa/cl/cd), ``cl0 [ns]`` or ``[ns, nb]`` (perf.cl at p = 1).
    ``user``: d, co, integ, tol, maxiter, relax. ``const`` as constants.m.
    Loads (optional, ``loads`` dict): twist_deg [ns] (blade.AeroTwst + pitch),
    r [ns], dr [ns], rpm [nt], rho.
    """

    def __init__(self, inp: dict, user: dict, const: dict | None = None, loads: dict | None = None):
        self.inp, self.user = inp, dict(user)
        self.const = dict(CONST if const is None else const)
        self.loads_in = loads
        q = inp["quarter"]
        self.nst, _, self.nt, self.nb = q.shape
        self.ns = self.nst - 1
        self.dt = 1.0 / user["hz"]
        self.p = 1
        self.T = self.Q = self.P = None
        self._initials()

    # ---------------------------------------------------------------- initials
    def _initials(self):
        """core/initials.m:37-152 (BEM's Cl given)."""
        inp, c = self.inp, self.const
        nst, ns, nb, nt = self.nst, self.ns, self.nb, self.nt
        infty = np.asarray(inp["infty"], np.float64)
        self.inftyM = np.sqrt(np.sum(infty ** 2, axis=1))
        # :43-113 preallocate and truncate each cell to p+1 (p) columns
        self.domain, self.vel, self.uind = {}, {}, {}
        self.shed, self.trail = {}, {}
        self.rc_s, self.rc_t, self.rce_s, self.rce_t = {}, {}, {}, {}
        self.len_s, self.len_t = {}, {}
        for j in range(1, nt + 1):
            d = np.zeros((nst, 3, j + 1, nb))
            d[:, :, 0, :] = inp["quarter"][:, :, j - 1, :]
            d[:, :, 1, :] = inp["trail"][:, :, j - 1, :]
            self.domain[j] = d
            self.vel[j] = np.broadcast_to(infty[j - 1][None, :, None, None], (nst, 3, j + 1, nb)).copy()
            self.uind[j] = np.zeros((nst, 3, j + 1, nb))
            self.shed[j] = np.zeros((ns, j + 1, nb))
            self.trail[j] = np.zeros((nst, j, nb))
        self.cl = np.zeros((ns, nt, nb))
        self.cd = np.zeros((ns, nt, nb))
        self.aoa = np.zeros((ns, nt, nb))
        cl0 = np.asarray(inp["cl0"], np.float64)
        if cl0.ndim == 1:
            cl0 = np.repeat(cl0[:, None], nb, axis=1)
        self.cl[:, 0, :] = cl0
        # :124-131 bound circulation, first trailing column, shed columns
        self.shed[1][:, 0, :] = 0.5 * self.inftyM[0] * np.asarray(inp["chord"])[:, None] * self.cl[:, 0, :]
        self.trail[1] = _diff_span(self.shed[1][:, 0, :])[:, None, :]
        self.shed[1][:, 1:, :] = _shed_rest(self.trail[1], ns)
        # :134-135 initial core radius per time step
        T0 = 2 * math.pi * inp["tip_rad"] / (12 * np.asarray(inp["tsr"], np.float64) * self.inftyM)
        self.r0 = np.sqrt(4 * c["alpha"] * c["nu"] * c["delta"] * T0)
        # :138-152 core, induced velocity on wake.domain{1}, forward Euler to p = 2
        self.vcore(1)
        self.uind[1] = self.induced(1)
        self.vel[1] = self.vel[1] + self.uind[1]
        self.fe(1)

    # ------------------------------------------------------------------ pieces
    def vcore(self, t):
        """core/vcore.m:30-51 at time index t."""
        c = self.const
        Re_s = np.abs(self.shed[t] / c["nu"])
        Re_t = np.abs(self.trail[t] / c["nu"])
        time = self.inp["time"][t - 1]
        r0 = self.r0[t - 1]
        self.rc_s[t] = r0 ** 2 + 4 * c["alpha"] * c["nu"] * (1 + c["a1"] * Re_s) * time
        self.rc_t[t] = r0 ** 2 + 4 * c["alpha"] * c["nu"] * (1 + c["a1"] * Re_t) * time
        self.rce_s[t] = self.rc_s[t].copy()
        self.rce_t[t] = self.rc_t[t].copy()
        d = self.domain[t]
        self.len_s[t] = self.filament_length(d[:-1], d[1:])
        self.len_t[t] = self.filament_length(d[:, :, 1:], d[:, :, :-1])
        self.filamentmod(t)

    @staticmethod
    def filament_length(F1, F2):
        """core/FilamentLength.m:27-44 -> [span, age, blade]."""
        x = F2[:, 0] - F1[:, 0]
        y = F2[:, 1] - F1[:, 1]
        z = F2[:, 2] - F1[:, 2]
        return np.sqrt(x ** 2 + y ** 2 + z ** 2)

    def filamentmod(self, t):
        """core/filamentmod.m:26-41: interior columns against the previous
        step's columns of the same index, lengths square-rooted again."""
        if t > 3:
            tn = np.sqrt(self.len_t[t][:, 1:-1])
            to = np.sqrt(self.len_t[t - 1][:, 1:])
            sn = np.sqrt(self.len_s[t][:, 1:-1])
            so = np.sqrt(self.len_s[t - 1][:, 1:])
            st_t = (tn - to) / to
            st_s = (sn - so) / so
            self.rce_t[t][:, 1:-1] = self.rc_t[t][:, 1:-1] * (1.0 / (1 + st_t))
            self.rce_s[t][:, 1:-1] = self.rc_s[t][:, 1:-1] * (1.0 / (1 + st_s))

    def _bs(self, t, P):
        d = self.domain[t]
        u = orc.c_eval(d[:-1], d[1:], P, self.shed[t][:, None], self.rce_s[t][:, None],
                       self.user["d"], self.user["co"])
        u = u + orc.c_eval(d[:, :, 1:], d[:, :, :-1], P, self.trail[t][:, None],
                           self.rce_t[t][:, None], self.user["d"], self.user["co"])
        return u

    def induced(self, t):
        """Shed + trailing induction at every node of wake.domain{t}."""
        return self._bs(t, self.domain[t])

    def fe(self, t):
        """numerical/fe.m:31."""
        self.domain[t + 1][:, :, 2:] = self.domain[t][:, :, 1:] + self.dt * self.vel[t][:, :, 1:]

    def ab2(self, t):
        """numerical/ab2.m:35-39 (t < 2: forward Euler)."""
        if t < 2:
            self.fe(t)
            return
        prev = np.concatenate([np.zeros((self.nst, 3, 1, self.nb)), self.vel[t - 1][:, :, 1:]], axis=2)
        self.domain[t + 1][:, :, 2:] = self.domain[t][:, :, 1:] + self.dt / 2 * (
            3 * self.vel[t][:, :, 1:] - prev)

    def ab4(self, t):
        """numerical/ab4.m:35-42 (t < 4: forward Euler)."""
        if t < 4:
            self.fe(t)
            return
        z = lambda k: np.zeros((self.nst, 3, k, self.nb))
        v = self.vel
        self.domain[t + 1][:, :, 2:] = self.domain[t][:, :, 1:] + self.dt / 24 * (
            55 * v[t][:, :, 1:]
            - 59 * np.concatenate([z(1), v[t - 1][:, :, 1:]], axis=2)
            + 37 * np.concatenate([z(2), v[t - 2][:, :, 1:]], axis=2)
            - 9 * np.concatenate([z(3), v[t - 3][:, :, 1:]], axis=2))

    def bookkeeping(self, t):
        """WInDS.m:131-140 (and numerical/pcc.m:43-49 for t = time + 1)."""
        self.shed[t][:, 0, :] = self.shed[t - 1][:, 0, :]
        self.trail[t][:, 0, :] = _diff_span(self.shed[t][:, 0, :])
        self.trail[t][:, 1:, :] = self.trail[t - 1]
        self.shed[t][:, 1:, :] = _shed_rest(self.trail[t], self.ns)

    def pcc(self, t):
        """numerical/pcc.m:37-75."""
        self.fe(t)
        if t > 2:
            self.bookkeeping(t + 1)
            self.vcore(t + 1)
            self.uind[t + 1] = self.induced(t + 1)
            self.vel[t + 1] = self.vel[t + 1] + self.uind[t + 1]
            self.domain[t + 1][:, :, 2:] = self.domain[t][:, :, 1:] + self.dt / 2 * (
                self.vel[t + 1][:, :, 2:] + self.vel[t][:, :, 1:])

    def kj(self, gamma, t):
        """core/KuttaJoukowski.m:173-298 (fixed point, no tower shadow)."""
        inp, ns, nb = self.inp, self.ns, self.nb
        cl = self.cl[:, t - 2, :].copy()
        cd = self.cd[:, t - 2, :].copy()
        self.shed[t][:, 0, :] = gamma
        P = inp["bound"][:, :, t - 1:t, :]
        u = self._bs(t, P)[:, :, 0, :]                                   # [ns,3,nb]
        bxn, byn, bzn = (inp[k][:, :, t - 1, :] for k in ("bxn", "byn", "bzn"))
        rot = np.stack([(bxn * u).sum(1), (byn * u).sum(1), (bzn * u).sum(1)], axis=1)
        vb = inp["vblade"][:, :, t - 1, :]
        tot = vb + rot
        Vinf = np.sqrt(np.sum(vb ** 2, axis=1))
        aoa = np.arctan2(-tot[:, 1], tot[:, 0]) * (180 / math.pi)
        nfoil = np.asarray(inp["nfoil"])
        for k, tab in enumerate(inp["tables"]):
            sel = nfoil == k + 1
            for m in range(nb):
                cl[sel, m] = interp1(tab["aoa"], tab["cl"], aoa[sel, m])
                cd[sel, m] = interp1(tab["aoa"], tab["cd"], aoa[sel, m])
        if np.any(np.isnan(cl)):
            raise KJDiverged("Diverging soln!!!")
        g = 0.5 * Vinf * np.asarray(inp["chord"])[:, None] * cl
        dg = g - self.shed[t][:, 0, :]
        self.shed[t][:, 0, :] = self.shed[t][:, 0, :] + self.user["relax"] * dg
        self.trail[t][:, 0, :] = _diff_span(self.shed[t][:, 0, :])
        self.shed[t][:, 1:, :] = _shed_rest(self.trail[t], ns)
        dg = dg / (np.abs(g) + 1)
        self.cl[:, t - 1, :], self.cd[:, t - 1, :], self.aoa[:, t - 1, :] = cl, cd, aoa
        return dg

    def kutta_joukowski(self, t):
        """core/KuttaJoukowski.m:42-49."""
        j, dg = 0, np.ones(1)
        while np.max(np.abs(dg)) > self.user["tol"] and j < self.user["maxiter"]:
            gamma = self.shed[t][:, 0, :].copy()
            dg = self.kj(gamma, t)
            j += 1
        return j

    # -------------------------------------------------------------------- loop
    def step(self):
        """One pass of WInDS.m:127-182 (p = 2, 3, ...); returns p."""
        p = self.p + 1
        if p > self.nt:
            raise IndexError("run is over")
        self.bookkeeping(p)
        self.vcore(p)
        self.uind[p] = self.induced(p)
        self.vel[p] = self.vel[p] + self.uind[p]
        integ = self.user["integ"]
        if p != self.nt:
            getattr(self, integ)(p)
        self.ctj = self.kutta_joukowski(p)
        if self.loads_in is not None:
            L = self.loads_in
            k = p - 1
            self.T, self.Q, self.P, _ = perform_ref.loads(
                self.cl[:, k, :], self.cd[:, k, :], self.aoa[:, k, :], self.inp["vblade"][:, :, k, :],
                L["twist_deg"], self.inp["chord"], L["r"], L["dr"], L["rpm"][k], L["rho"])
        self.p = p
        return p

    @property
    def bound(self):
        return self.shed[self.p][:, 0, :]
