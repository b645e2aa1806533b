"""Seeded synthetic helical rotor wakes in WInDS's own array layout.

WInDS stores every per-node and per-filament quantity as a MATLAB column-major
4-D double array shaped ``[span, component, age, blade]``:

* wake nodes ``wake.domain{p}``: ``[nst, 3, na, nb]`` with ``na = p + 1`` age
  columns (``core/initials.m:44-51,84-87``);
* shed filaments ``F1 = dom(1:end-1,:,:,:)``, ``F2 = dom(2:end,:,:,:)``:
  ``[ns, 3, na, nb]`` (``WInDS.m:150``);
* trailing filaments ``F1 = dom(:,:,2:end,:)``, ``F2 = dom(:,:,1:end-1,:)``:
  ``[nst, 3, na-1, nb]`` (``WInDS.m:153``);
* circulation / squared core radius: ``[n, 1, m, nb]``.

Python keeps the same shapes as Fortran-ordered ``numpy`` arrays, so
``arr.ravel(order="F")`` is the byte image MATLAB hands to a MEX file.

The circulation bookkeeping follows ``WInDS.m:131-140``: the trailing column
built from bound circulation ``G`` is ``diff([0; G; 0])`` and the shed columns
are ``diff(cat(3, cumsum(trail(1:end-1)), 0), 1, 3)`` behind the bound column.
The core model is the age-based Ramasamy-Leishman growth
``rc^2 = rc0^2 + 4 alpha delta nu age`` (squared radius, as ``BiotSavart``
expects it: ``core/BiotSavart.m:13``).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

ALPHA_RL = 1.25643  # Ramasamy-Leishman alpha, core/constants.m:22


@dataclasses.dataclass
class RotorCase:
    """One rotor and its helical wake. Defaults: the 3.2k-target case
    (3 blades, R = 63 m, 17 cosine-spaced nodes from 1.5 m, 60 steps of 10 deg,
    12.1 rpm, U = 11.4 m/s)."""

    nb: int = 3
    R: float = 63.0
    r_root: float = 1.5
    nst: int = 17
    nsteps: int = 60
    dpsi_deg: float = 10.0
    omega_rpm: float = 12.1
    U: float = 11.4
    yaw_deg: float = 0.0
    shear: float = 0.0
    hub_height: float = 90.0
    jitter: float = 0.05
    gamma_peak: float = 80.0
    gamma_noise: float = 0.02
    rc0: float = 0.1
    delta: float = 100.0
    nu: float = 1.5e-5
    seed: int = 0

    @property
    def omega(self) -> float:
        """Rotor speed in rad/s."""
        return self.omega_rpm * 2.0 * math.pi / 60.0

    @property
    def dt(self) -> float:
        """Time step: one azimuth increment at the rotor speed."""
        return math.radians(self.dpsi_deg) / self.omega

    @property
    def ns(self) -> int:
        return self.nst - 1

    @property
    def na(self) -> int:
        return self.nsteps + 1

    def counts(self) -> dict:
        nt = self.nst * self.na * self.nb
        nll = self.ns * self.nb
        nshed = self.ns * self.na * self.nb
        ntrail = self.nst * (self.na - 1) * self.nb
        return dict(wake_targets=nt, ll_targets=nll, shed=nshed, trail=ntrail,
                    targets=nt + nll, filaments=nshed + ntrail,
                    interactions=(nt + nll) * (nshed + ntrail))


def cosine_nodes(r_root: float, R: float, n: int) -> np.ndarray:
    """Cosine-spaced radial node positions from ``r_root`` to ``R``."""
    i = np.arange(n, dtype=np.float64)
    return r_root + (R - r_root) * 0.5 * (1.0 - np.cos(math.pi * i / (n - 1)))


def elliptic_bound(case: RotorCase, r_mid: np.ndarray) -> np.ndarray:
    """Elliptical spanwise bound circulation at station midpoints."""
    half = 0.5 * (case.R - case.r_root)
    mid = 0.5 * (case.R + case.r_root)
    s = np.clip((r_mid - mid) / half, -1.0, 1.0)
    return case.gamma_peak * np.sqrt(1.0 - s * s)


def trail_from_bound(G: np.ndarray) -> np.ndarray:
    """``diff([0; G; 0])`` along span for every (age, blade) column.
    ``G``: ``[ns, m, nb]`` -> ``[nst, m, nb]`` (``WInDS.m:133-134``)."""
    z = np.zeros((1,) + G.shape[1:])
    return np.diff(np.concatenate([z, G, z], axis=0), axis=0)


def shed_from_trail(trail: np.ndarray) -> np.ndarray:
    """Shed columns 2:end from the trailing columns (``WInDS.m:139-140``):
    ``diff(cat(3, cumsum(trail(1:end-1,:,:,:),1), 0), 1, 3)``.
    ``trail``: ``[nst, m, nb]`` -> ``[ns, m, nb]``."""
    c = np.cumsum(trail[:-1], axis=0)
    z = np.zeros((c.shape[0], 1, c.shape[2]))
    return np.diff(np.concatenate([c, z], axis=1), axis=1)


def core_sq(case: RotorCase, age_s: np.ndarray) -> np.ndarray:
    """Squared core radius after ``age_s`` seconds."""
    return case.rc0 ** 2 + 4.0 * ALPHA_RL * case.delta * case.nu * age_s


def make_wake(case: RotorCase) -> dict:
    """Build node positions, circulations and squared cores for one case.

    Returns a dict of Fortran-ordered float64 arrays in WInDS layout:
    ``dom [nst,3,na,nb]``, ``ll [ns,3,1,nb]`` (lifting-line points = bound
    filament midpoints), ``gamma_shed [ns,1,na,nb]``, ``gamma_trail
    [nst,1,na-1,nb]``, ``rc_shed``/``rc_trail`` (squared radii, same shapes),
    ``bound`` ``[ns, na, nb]`` (the bound-circulation history)."""
    rng = np.random.Generator(np.random.PCG64(case.seed))
    nst, na, nb, ns = case.nst, case.na, case.nb, case.ns
    r = cosine_nodes(case.r_root, case.R, nst)
    tau = np.arange(na, dtype=np.float64) * case.dt
    psi_b = 2.0 * math.pi * np.arange(nb) / nb
    # helix in the rotor frame: x axial (downwind), y/z in the rotor plane
    psi = psi_b[None, None, :] - case.omega * tau[None, :, None]       # [1, na, nb]
    rr = r[:, None, None]
    yr = rr * np.cos(psi)
    zr = rr * np.sin(psi) + 0.0 * tau[None, :, None]
    # rotor yawed about the vertical (z) axis; wake convects along +x
    yaw = math.radians(case.yaw_deg)
    xr_plane = -yr * math.sin(yaw)
    yr_plane = yr * math.cos(yaw)
    height = case.hub_height + zr
    speed = case.U * np.power(np.maximum(height, 1.0) / case.hub_height, case.shear)
    x = xr_plane + speed * tau[None, :, None]
    y = yr_plane + 0.0 * x
    z = zr + 0.0 * x
    dom = np.stack([x, y, z], axis=1)                                  # [nst,3,na,nb]
    dom = dom + rng.normal(0.0, case.jitter, size=dom.shape)
    dom = np.asfortranarray(dom)

    r_mid = 0.5 * (r[1:] + r[:-1])
    G = elliptic_bound(case, r_mid)[:, None, None] * (
        1.0 + case.gamma_noise * rng.standard_normal((ns, na, nb)))  # [ns, na, nb]
    trail = trail_from_bound(G[:, : na - 1, :])                        # [nst, na-1, nb]
    shed = np.empty((ns, na, nb))
    shed[:, 0, :] = G[:, 0, :]
    shed[:, 1:, :] = shed_from_trail(trail)

    rc_shed = core_sq(case, tau)[None, :, None] * np.ones((ns, 1, nb))
    tmid = 0.5 * (tau[1:] + tau[:-1])
    rc_trail = core_sq(case, tmid)[None, :, None] * np.ones((nst, 1, nb))

    ll = 0.5 * (dom[:-1, :, 0:1, :] + dom[1:, :, 0:1, :])
    f = np.asfortranarray
    return dict(
        dom=dom,
        ll=f(ll),
        gamma_shed=f(shed[:, None, :, :]),
        gamma_trail=f(trail[:, None, :, :]),
        rc_shed=f(rc_shed[:, None, :, :]),
        rc_trail=f(rc_trail[:, None, :, :]),
        bound=G,
        case=case,
    )


def shed_filaments(dom: np.ndarray):
    """``F1, F2`` of the shed call (``WInDS.m:150``)."""
    return np.asfortranarray(dom[:-1]), np.asfortranarray(dom[1:])


def trail_filaments(dom: np.ndarray):
    """``F1, F2`` of the trailing call (``WInDS.m:153``)."""
    return np.asfortranarray(dom[:, :, 1:]), np.asfortranarray(dom[:, :, :-1])


def flat_filaments(w: dict):
    """All shed + trailing filaments flattened in MATLAB order:
    ``(x1 [nf,3], x2 [nf,3], gamma [nf], rc [nf])``, shed first."""
    out = []
    for (F1, F2), g, rc in ((shed_filaments(w["dom"]), w["gamma_shed"], w["rc_shed"]),
                            (trail_filaments(w["dom"]), w["gamma_trail"], w["rc_trail"])):
        x1 = np.stack([F1[:, c].ravel(order="F") for c in range(3)], axis=1)
        x2 = np.stack([F2[:, c].ravel(order="F") for c in range(3)], axis=1)
        out.append((x1, x2, g.ravel(order="F"), rc.ravel(order="F")))
    return tuple(np.concatenate([o[i] for o in out]) for i in range(4))


def flat_points(P: np.ndarray) -> np.ndarray:
    """Targets ``[n, 3]`` in MATLAB order from a ``[ns,3,nt,nb]`` array."""
    return np.stack([P[:, c].ravel(order="F") for c in range(3)], axis=1)


def large_case(seed: int = 1) -> RotorCase:
    """3 blades x 41 nodes x 720 steps at 1 deg (two revolutions)."""
    return RotorCase(nst=41, nsteps=720, dpsi_deg=1.0, seed=seed)


def near_singular_targets(x1, x2, rc_sq, n, rng, frac_rc=0.5):
    """``n`` points each within ``frac_rc * rc`` of a randomly chosen
    segment (random station along it, random perpendicular offset)."""
    idx = rng.integers(0, x1.shape[0], size=n)
    a, b = x1[idx], x2[idx]
    Lv = b - a
    t = rng.uniform(0.05, 0.95, size=n)[:, None]
    base = a + t * Lv
    rnd = rng.standard_normal((n, 3))
    Lhat = Lv / np.maximum(np.linalg.norm(Lv, axis=1, keepdims=True), 1e-300)
    perp = rnd - np.sum(rnd * Lhat, axis=1, keepdims=True) * Lhat
    perp /= np.maximum(np.linalg.norm(perp, axis=1, keepdims=True), 1e-300)
    dist = rng.uniform(0.05, frac_rc, size=n)[:, None] * np.sqrt(rc_sq[idx])[:, None]
    return base + dist * perp
