"""FP64 oracle of the Kutta-Joukowski fixed point (test infrastructure).

Restates ``core/KuttaJoukowski.m:42-49`` (the ``'fixed'`` loop) and its
``kj()`` iteration (``:173-298``): Biot-Savart of the shed and trailing
filaments onto the lifting-line points (``:215-227``), transform to the blade
frame (``:241-246``), ``aoa = atan2(-v, u)`` in degrees (``:258``), linear
``interp1`` of Cl and Cd with NaN outside the table (``:262-269``), the
divergence error on NaN Cl (``:272-274``), ``Γ = ½ |V| c Cl`` (``:277``), the
relaxed update (``:281``), the trailing/shed update (``:285-288``) and the
relative residual ``dg/(|Γ|+1)`` (``:290``). The cores stay those of the
step's ``vcore`` call; they are not recomputed inside the loop, as in kj().
"""
from __future__ import annotations

import numpy as np

import oracle as orc
import wake_ref


class KJDiverged(RuntimeError):
    pass


def interp1(x, y, xi):
    """MATLAB ``interp1(x, y, xi)``: linear, NaN outside ``[x(1), x(end)]``."""
    out = np.interp(xi, x, y)
    out = np.where((xi < x[0]) | (xi > x[-1]) | np.isnan(xi), np.nan, out)
    return out


def kj_solve(kj, s, dom, trail_prev, rcs, rct, bound0, relax=0.25, tol=1e-6, maxiter=30,
             d="visc2", co=1000.0):
    """Fixed-point iteration at step ``s`` of one case. ``kj``: the dict of
    ``synth.make_kj_case``. Returns ``(bound, iterations, residual, cl, cd, aoa)``."""
    ll = kj["ll"][:, :, s:s + 1, :]                  # [ns,3,1,nb]
    bxn, byn, bzn = (kj[k][:, :, s, :] for k in ("bxn", "byn", "bzn"))
    vb = kj["vblade"][:, :, s, :]
    chord = kj["chord"][:, None]
    bound = bound0.copy()
    j, dg = 0, np.ones_like(bound)
    F1s, F2s = dom[:-1], dom[1:]
    F1t, F2t = dom[:, :, 1:], dom[:, :, :-1]
    cl = cd = aoa = None
    while np.max(np.abs(dg)) > tol and j < maxiter:
        shed, trail = wake_ref.bookkeeping(bound, trail_prev)
        u = orc.c_eval(F1s, F2s, ll, shed[:, None], rcs[:, None], d, co)
        u = u + orc.c_eval(F1t, F2t, ll, trail[:, None], rct[:, None], d, co)
        u = u[:, :, 0, :]                            # [ns,3,nb]
        rotv = np.stack([(bxn * u).sum(1), (byn * u).sum(1), (bzn * u).sum(1)], axis=1)
        tot = vb + rotv
        Vinf = np.sqrt((vb ** 2).sum(1))             # [ns,nb]
        aoa = np.arctan2(-tot[:, 1], tot[:, 0]) * (180.0 / np.pi)
        foil = kj["foil"]
        cl = np.empty_like(aoa)
        cd = np.empty_like(aoa)
        offs = np.concatenate([[0], np.cumsum(kj["foil_points"])])
        for f in range(len(kj["foil_points"])):
            a = kj["aoa"][offs[f]:offs[f + 1]]
            sel = foil == f
            cl[sel] = interp1(a, kj["cl"][offs[f]:offs[f + 1]], aoa[sel])
            cd[sel] = interp1(a, kj["cd"][offs[f]:offs[f + 1]], aoa[sel])
        if np.any(np.isnan(cl)):
            raise KJDiverged("Diverging soln!!!")
        gamma = 0.5 * Vinf * chord * cl
        dgv = gamma - bound
        bound = bound + relax * dgv
        dg = dgv / (np.abs(gamma) + 1.0)
        j += 1
    return bound, j, float(np.max(np.abs(dg))), cl, cd, aoa


class KJWakeRef(wake_ref.WakeRef):
    """The step oracle with the lifting line: after the convection of step
    ``p`` the fixed point runs on ``wake.domain{p}`` with the step's cores and
    the converged bound column re-forms the step's Γ (kj(), :285-288), which
    the next step's bookkeeping carries on (WInDS.m:131-140)."""

    def __init__(self, case, kj, relax=0.25, tol=1e-6, maxiter=30, **kw):
        super().__init__(case, **kw)
        self.kj, self.relax, self.tol, self.maxiter = kj, relax, tol, maxiter

    def _before_commit(self, s):
        out = kj_solve(self.kj, s, self.dom, self.trail_prev, self.rcs, self.rct, self.bound,
                       self.relax, self.tol, self.maxiter, self.d, self.co)
        self.bound, self.kj_iters, self.kj_res, self.cl, self.cd, self.aoa = out
        self.shed, self.trail = wake_ref.bookkeeping(self.bound, self.trail_prev)
        kj = self.kj
        if "r_station" in kj:  # rotor loads of the step (postproc/perform.m)
            import perform_ref
            theta = np.degrees(kj["twist"])
            if kj.get("pitch") is not None:  # per step and blade (perform.m:22-33)
                theta = theta[:, None] + np.asarray(kj["pitch"])[s][None, :]
            self.T, self.Q, self.P, _ = perform_ref.loads(
                self.cl, self.cd, self.aoa, kj["vblade"][:, :, s, :], theta,
                kj["chord"], kj["r_station"], kj["dr_station"], kj["rpm"][s], kj["rho"])
