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
RHO = 1.225  # air density, kg/m^3


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


# ----------------------------------------------------------------- time stepping
def blade_geometry(case: RotorCase):
    """Cosine-spaced node radii, linear chord 3.5 -> 1.4 m and twist 13 -> 0 deg
    from root to tip (the synthetic blade of the configurations)."""
    r = cosine_nodes(case.r_root, case.R, case.nst)
    s = (r - case.r_root) / (case.R - case.r_root)
    chord = 3.5 + (1.4 - 3.5) * s
    twist = np.radians(13.0 * (1.0 - s))
    return r, chord, twist


def blade_nodes(case: RotorCase, t: float, pitch_deg: float = 0.0):
    """Quarter-chord and trailing-edge nodes ``[nst, 3, nb]`` at time ``t``
    (rigid rotor turning at ``case.omega`` about the x axis, yawed about z)."""
    r, chord, twist = blade_geometry(case)
    psi = 2.0 * np.pi * np.arange(case.nb) / case.nb + case.omega * t      # [nb]
    cp, sp = np.cos(psi)[None, :], np.sin(psi)[None, :]
    rr = r[:, None]
    # rotor frame: x axial (downwind), y/z in the plane; tangential t = d/dpsi
    q = np.stack([np.zeros_like(rr * cp), rr * cp, rr * sp], axis=1)       # [nst,3,nb]
    tang = np.stack([np.zeros_like(cp + 0 * rr), -sp + 0 * rr, cp + 0 * rr], axis=1)
    th = (twist + np.radians(pitch_deg))[:, None]
    d = -np.cos(th)[:, None, :] * tang
    d[:, 0, :] += np.sin(th)
    te = q + 0.75 * chord[:, None, None] * d
    yaw = np.radians(case.yaw_deg)

    def rot(v):
        x, y, z = v[:, 0], v[:, 1], v[:, 2]
        return np.stack([x * np.cos(yaw) - y * np.sin(yaw), x * np.sin(yaw) + y * np.cos(yaw), z], axis=1)

    return rot(q), rot(te)


def make_wake_case(case: RotorCase, nsteps: int, t0: float = 0.0, jitter: float = 0.0,
                   a1: float = 0.0, pitch_deg: float = 0.0) -> dict:
    """Initial state, kinematics and wind of one rotor for the device time step.

    The wake keeps ``na = case.nsteps + 1`` age columns: column 0 the
    quarter-chord nodes, column 1 the trailing-edge nodes at ``t0``, column
    ``j >= 2`` the trailing-edge node of ``j - 1`` steps earlier convected by
    the freestream. Γ history as in :func:`make_wake`; core model: age form
    with the configurations' rc0, delta, nu."""
    rng = np.random.Generator(np.random.PCG64(case.seed))
    nst, nb, na, ns, dt = case.nst, case.nb, case.na, case.ns, case.dt
    quarter = np.zeros((nst, 3, nsteps, nb))
    trailing = np.zeros((nst, 3, nsteps, nb))
    for s in range(nsteps):
        quarter[:, :, s, :], trailing[:, :, s, :] = blade_nodes(case, t0 + s * dt, pitch_deg)
    dom = np.zeros((nst, 3, na, nb))
    q0, te0 = blade_nodes(case, t0, pitch_deg)
    dom[:, :, 0, :], dom[:, :, 1, :] = q0, te0
    for j in range(2, na):
        age = (j - 1) * dt
        _, te = blade_nodes(case, t0 - age, pitch_deg)
        height = case.hub_height + te[:, 2, :]
        speed = case.U * np.power(np.maximum(height, 1.0) / case.hub_height, case.shear)
        te[:, 0, :] += speed * age
        dom[:, :, j, :] = te
    if jitter > 0:
        dom[:, :, 2:, :] += rng.normal(0.0, jitter, size=dom[:, :, 2:, :].shape)
    r = cosine_nodes(case.r_root, case.R, nst)
    r_mid = 0.5 * (r[1:] + r[:-1])
    G = elliptic_bound(case, r_mid)[:, None, None] * (
        1.0 + case.gamma_noise * rng.standard_normal((ns, na, nb)))
    trail = trail_from_bound(G[:, : na - 1, :])          # [nst, na-1, nb]
    wind = np.zeros((3, nsteps))
    wind[0, :] = case.U
    f = np.asfortranarray
    return dict(nst=nst, nb=nb, na=na, nsteps=nsteps, dt=dt, t0=t0,
                quarter=f(quarter), trailing=f(trailing), wind=f(wind), shear=case.shear,
                hub_height=case.hub_height, core_mode=1, r0=case.rc0, rc0=case.rc0,
                alpha=ALPHA_RL, nu=case.nu, a1=a1, delta=case.delta,
                dom=f(dom), bound=f(G[:, 0, :]), trail_gamma=f(trail))


def batch_cases(n: int, seed: int = 0, steps_range=(60, 720), nodes_range=(17, 41),
                U_range=(5.0, 25.0), tsr_range=(4.0, 10.0), yaw_range=(0.0, 30.0),
                shear_range=(0.0, 0.3), dpsi_deg=None):
    """``n`` uneven rotor cases drawn uniformly from the seed: wake steps,
    span nodes, wind speed, tip-speed ratio, yaw and shear exponent. Without
    ``dpsi_deg`` every wake spans two revolutions (azimuth step 720/steps deg)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for k in range(n):
        U = float(rng.uniform(*U_range))
        tsr = float(rng.uniform(*tsr_range))
        omega = tsr * U / 63.0
        nst = int(rng.integers(nodes_range[0], nodes_range[1] + 1))
        steps = int(rng.integers(steps_range[0], steps_range[1] + 1))
        out.append(RotorCase(nst=nst, nsteps=steps,
                             dpsi_deg=dpsi_deg if dpsi_deg else 720.0 / steps,
                             omega_rpm=omega * 60 / (2 * np.pi), U=U,
                             yaw_deg=float(rng.uniform(*yaw_range)),
                             shear=float(rng.uniform(*shear_range)), seed=seed * 1000 + k))
    return out


# ----------------------------------------------------------- lifting line (KJ)
def synthetic_polar(step_deg: float = 0.25):
    """Airfoil table on [-180, 180] deg: Cl = 2 pi sin(a) cos(a) up to the
    12 deg stall, then 1.2 sin(2a) (continued on both signs); Cd = 0.008 +
    0.6 sin^2(a)."""
    a = np.arange(-180.0, 180.0 + step_deg / 2, step_deg)
    r = np.radians(a)
    cl = np.where(np.abs(a) <= 12.0, 2 * np.pi * np.sin(r) * np.cos(r), 1.2 * np.sin(2 * r))
    cd = 0.008 + 0.6 * np.sin(r) ** 2
    return a, cl, cd


def make_kj_case(case: RotorCase, nsteps: int, t0: float = 0.0, pitch_deg: float = 0.0,
                 root_cut: float = 0.0) -> dict:
    """Lifting-line inputs of ``core/KuttaJoukowski.m:173-298`` for every step:
    ``ll`` (pos.bound: quarter-chord midpoints), blade-frame unit vectors
    ``bxn`` (chord, leading to trailing edge), ``byn``, ``bzn`` (radial), the
    blade-frame velocity ``vblade`` (wind minus blade motion, vel.blade),
    chord, one airfoil for every station (``synthetic_polar``)."""
    nst, nb, ns = case.nst, case.nb, case.ns
    r, chord_n, twist_n = blade_geometry(case)
    rm = 0.5 * (r[1:] + r[:-1])
    s = (rm - case.r_root) / (case.R - case.r_root)
    chord = 3.5 + (1.4 - 3.5) * s
    th = np.radians(13.0 * (1.0 - s) + pitch_deg)
    yaw = np.radians(case.yaw_deg)

    def rot(v):  # yaw about z, v [..., 3]
        x, y, z = v[..., 0], v[..., 1], v[..., 2]
        return np.stack([x * np.cos(yaw) - y * np.sin(yaw), x * np.sin(yaw) + y * np.cos(yaw), z], axis=-1)

    shape = (ns, 3, nsteps, nb)
    out = {k: np.zeros(shape) for k in ("ll", "bxn", "byn", "bzn", "vblade")}
    for st in range(nsteps):
        t = t0 + st * case.dt
        q, _ = blade_nodes(case, t, pitch_deg)
        out["ll"][:, :, st, :] = 0.5 * (q[1:] + q[:-1])
        psi = 2.0 * np.pi * np.arange(nb) / nb + case.omega * t            # [nb]
        rhat = np.stack([np.zeros(nb), np.cos(psi), np.sin(psi)], axis=-1)  # [nb, 3]
        that = np.stack([np.zeros(nb), -np.sin(psi), np.cos(psi)], axis=-1)
        xhat = np.array([1.0, 0.0, 0.0])
        ct, sn = np.cos(th)[:, None, None], np.sin(th)[:, None, None]
        d = -ct * that[None] + sn * xhat[None, None]                          # chord LE->TE
        n = sn * that[None] + ct * xhat[None, None]
        bx, by, bz = rot(d), rot(-n), rot(np.broadcast_to(rhat[None], d.shape))
        # relative wind at the station: freestream (with shear) minus blade velocity
        pts = out["ll"][:, :, st, :].transpose(0, 2, 1)                      # [ns, nb, 3]
        h = np.maximum(case.hub_height + pts[..., 2], 1.0) / case.hub_height
        w = np.zeros_like(pts)
        w[..., 0] = case.U * h ** case.shear
        vb = rot(case.omega * rm[:, None, None] * that[None])                # blade velocity
        wr = w - vb
        out["bxn"][:, :, st, :] = bx.transpose(0, 2, 1)
        out["byn"][:, :, st, :] = by.transpose(0, 2, 1)
        out["bzn"][:, :, st, :] = bz.transpose(0, 2, 1)
        out["vblade"][:, :, st, :] = np.stack([(wr * bx).sum(-1), (wr * by).sum(-1),
                                               (wr * bz).sum(-1)], axis=1)
    a, cl, cd = synthetic_polar()
    foil = np.zeros(ns, dtype=np.int32)
    foil_points = [a.size]
    if root_cut > 0:
        # cylindrical root sections (no lift, Cd 0.5) inside r/R < root_cut
        foil[rm / case.R < root_cut] = 1
        ac = np.array([-180.0, 180.0])
        a, cl, cd = np.concatenate([a, ac]), np.concatenate([cl, [0.0, 0.0]]), np.concatenate([cd, [0.5, 0.5]])
        foil_points.append(2)
    f = np.asfortranarray
    res = {k: f(v) for k, v in out.items()}
    steps = t0 + case.dt * np.arange(nsteps)
    azimuth = 2.0 * np.pi * np.arange(nb)[None, :] / nb + case.omega * steps[:, None]  # [nsteps, nb]
    res.update(chord=chord, foil=foil, foil_points=np.array(foil_points, dtype=np.int32),
               aoa=a, cl=cl, cd=cd, twist_deg=np.degrees(th), r_over_R=rm / case.R,
               chord_over_R=chord / case.R, twist=th.copy(), azimuth=f(azimuth),
               r_station=rm.copy(), dr_station=np.diff(r), rpm=np.full(nsteps, case.omega_rpm),
               rho=RHO)
    return res


def kj_features(kj: dict, s: int, bound, bound_last=None, uind=None, bound_last2=None) -> np.ndarray:
    """Inputs of the bound-circulation MLP at step ``s`` (rows i + ns*b), the
    device's feature order, as float32: r/R, chord/R, twist, sin/cos azimuth,
    local inflow in the blade frame (vblade plus ``uind`` [ns,3,nb], the
    previous step's induced velocity at the lifting line, rotated with
    bxn/byn/bzn; zero when None), bound circulation, its change since
    ``bound_last`` and the change from ``bound_last2`` to ``bound_last``
    (zero when None)."""
    ns, _, _, nb = kj["vblade"].shape
    az = kj["azimuth"][s]                                   # [nb]
    vb = kj["vblade"][:, :, s, :].copy()                    # [ns, 3, nb]
    if uind is not None:
        for a, key in enumerate(("bxn", "byn", "bzn")):
            vb[:, a, :] += (kj[key][:, :, s, :] * uind).sum(1)
    bound = np.asarray(bound, dtype=np.float64)
    last = np.asarray(bound_last, dtype=np.float64) if bound_last is not None else bound
    d = bound - last
    d2 = last - (np.asarray(bound_last2, dtype=np.float64) if bound_last2 is not None else last)
    cols = [np.repeat(kj["r_over_R"][:, None], nb, 1), np.repeat(kj["chord_over_R"][:, None], nb, 1),
            np.repeat(kj["twist"][:, None], nb, 1), np.repeat(np.sin(az)[None, :], ns, 0),
            np.repeat(np.cos(az)[None, :], ns, 0), vb[:, 0], vb[:, 1], vb[:, 2], bound, d, d2]
    return np.stack([c.ravel(order="F") for c in cols], axis=1).astype(np.float32)


def rotor_series(case: RotorCase, nsteps: int, pitch_deg: float = 0.0, tilt_deg: float = 5.0,
                 precone_deg: float = -2.5, nac_yaw_deg: float = 0.0, platform_motion: bool = False,
                 seed: int = 0) -> dict:
    """Turbine time series and geometry in the form of core/kinematics.m's
    inputs (fastout.*, blade.*, turbine.*): the synthetic blade (cosine
    trailing nodes, stations at their midpoints, chord 3.5 -> 1.4 m, twist
    13 -> 0 deg), constant rotor speed, blade pitch with a small per-blade
    oscillation, nacelle yaw, and (optionally) a seeded platform motion."""
    rng = np.random.Generator(np.random.PCG64(seed))
    r, chord, twist = blade_geometry(case)
    rm = 0.5 * (r[1:] + r[:-1])
    s = (rm - case.r_root) / (case.R - case.r_root)
    t = case.dt * np.arange(nsteps)
    az = np.degrees(case.omega * t)
    pitch = pitch_deg + 0.5 * np.sin(2 * np.pi * 0.1 * t[:, None] + np.arange(case.nb)[None, :])
    ptfm = np.zeros((nsteps, 6))
    if platform_motion:
        amp = rng.uniform(0.2, 1.0, 6) * np.array([1.0, 0.5, 0.3, 2.0, 3.0, 1.5])
        ph = rng.uniform(0, 2 * np.pi, 6)
        ptfm = amp[None, :] * np.sin(2 * np.pi * 0.05 * t[:, None] + ph[None, :])
    wind = np.zeros((nsteps, 3))
    wind[:, 0] = case.U
    return dict(time=t, azimuth=az, pitch=pitch, nac_yaw=np.full(nsteps, nac_yaw_deg), ptfm=ptfm,
                wind=wind, r_trail=r, chord_trail=chord, twist_trail=np.degrees(twist), r_nodes=rm,
                chord=3.5 + (1.4 - 3.5) * s, twist=13.0 * (1.0 - s),
                precone=np.full(case.nb, precone_deg), overhang=-5.0, shaft_tilt=tilt_deg,
                tower_ht=87.6, twr2shft=1.96, ptfm_ref=0.0)
