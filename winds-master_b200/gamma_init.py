"""The learned start value of the Kutta-Joukowski iteration.

The plain solver (the batched device time step with the lifting-line fixed
point of ``core/KuttaJoukowski.m:42-49``, started from the previous step's
bound circulation as ``WInDS.m:131`` does) generates pairs (station state,
converged bound circulation); the MLP of ``winds_mlp.h`` learns the change
``Gamma_conv - Gamma_prev`` from the state and then starts each step's
iteration at ``Gamma_prev + out_scale * network(state)``; with the
extrapolated base (the default of ``study``) it learns the residual of the
linear extrapolation instead and starts at ``Gamma_prev + dGamma_prev +
out_scale * network(state)``. The iteration still
runs to the same tolerance, so converged results are unchanged and only
iterations (each one two Biot-Savart calls in the reference: shed and
trailing filaments onto the lifting line) are saved.

Operating points: 3 blades, R = 63 m, 41 span nodes, 10 deg per step, wind
speed U in [5, 25] m/s, blade pitch in [0, 15] deg, yaw in [0, 30] deg and
tip-speed ratio in [5, 9] (rotor speed TSR U / R), drawn from a seed;
synthetic blade and polar (chord 3.5 -> 1.4 m, twist 13 -> 0 deg, Cl =
2 pi sin a cos a to the 12 deg stall, then 1.2 sin 2a; Cd = 0.008 +
0.6 sin^2 a) with cylindrical root sections (Cl = 0) inside r/R < 0.2.

Features (device-computed, ``winds_wake_get_kj_features``): r/R, chord/R,
twist, sin and cos of the azimuth, the local inflow in the blade frame
(kinematic inflow plus the previous step's induced velocity at the lifting
line), the previous bound circulation, its change over the previous step and
the change over the step before that (with which the network can form a
second-order extrapolation).
Training pairs come only from (case, step) whose plain iteration converged,
and only from the stations the start value applies to (``start_rows``):
lifting stations whose previous converged AoA is inside their table's stall
bounds. A station whose airfoil table has no lift (the cylinder root
sections) converges to Gamma = 0, and any start there but the previous value
costs iterations (the relaxed iteration damps it by only 1 - relax per
iteration); a station past stall can have more than one fixed point, and the
previous value keeps the branch it is on.
"""
from __future__ import annotations

import dataclasses
import time

import numpy as np

from . import synth
from .mlp import Mlp
from .wake import WakeBatch

N_FEATURES = 11


@dataclasses.dataclass
class OperatingPoint:
    case: synth.RotorCase
    pitch_deg: float


ROOT_CUT = 0.2


def operating_points(n: int, seed: int, nst: int = 41, wake_steps: int = 36,
                     dpsi_deg: float = 10.0, U=(5.0, 25.0), pitch=(0.0, 15.0), yaw=(0.0, 30.0),
                     tsr=(5.0, 9.0), shear: float = 0.0):
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for k in range(n):
        u = float(rng.uniform(*U))
        omega = float(rng.uniform(*tsr)) * u / 63.0
        c = synth.RotorCase(nst=nst, nsteps=wake_steps, dpsi_deg=dpsi_deg, U=u,
                            omega_rpm=omega * 60.0 / (2.0 * np.pi),
                            yaw_deg=float(rng.uniform(*yaw)), shear=shear,
                            seed=seed * 10007 + k, jitter=0.0)
        out.append(OperatingPoint(c, float(rng.uniform(*pitch))))
    return out


STALL_MARGIN = 2.0  # degrees inside the stall bounds (kj_kernels.cu: kStallMargin)


def lifting_stations(kj: dict) -> np.ndarray:
    """[ns] bool: the stations whose airfoil table has some Cl != 0."""
    offs = np.concatenate([[0], np.cumsum(kj["foil_points"])])
    lift = np.array([np.any(np.asarray(kj["cl"])[offs[f]:offs[f + 1]] != 0.0)
                     for f in range(len(kj["foil_points"]))])
    return lift[np.asarray(kj["foil"])]


def stall_bounds(kj: dict) -> np.ndarray:
    """[ns, 2]: per station, the AoA (deg) of its table's lowest Cl in
    [-45, 0] and highest Cl in [0, 45] deg, as the engine computes them."""
    offs = np.concatenate([[0], np.cumsum(kj["foil_points"])])
    out = []
    for f in range(len(kj["foil_points"])):
        a = np.asarray(kj["aoa"])[offs[f]:offs[f + 1]]
        c = np.asarray(kj["cl"])[offs[f]:offs[f + 1]]
        hi, lo = (a >= 0) & (a <= 45), (a <= 0) & (a >= -45)
        ahi = a[hi][np.argmax(c[hi])] if hi.any() else 45.0
        alo = a[lo][np.argmin(c[lo])] if lo.any() else -45.0
        out.append((alo, ahi))
    return np.asarray(out)[np.asarray(kj["foil"])]


def start_rows(kj: dict, nb: int, aoa_prev) -> np.ndarray:
    """[ns*nb] bool (rows i + ns*b): where the engine's start value applies
    -- lifting stations whose last converged AoA ``aoa_prev`` [ns, nb] lies
    inside their table's stall bounds less STALL_MARGIN; elsewhere the start
    is the previous step's circulation."""
    sb = stall_bounds(kj)
    ap = np.asarray(aoa_prev, np.float64)
    inside = (ap > sb[:, :1] + STALL_MARGIN) & (ap < sb[:, 1:] - STALL_MARGIN)
    return (inside & lifting_stations(kj)[:, None]).ravel(order="F")


def build(points, run_steps: int, root_cut: float = ROOT_CUT):
    """Wake and lifting-line inputs of every point for ``run_steps`` steps."""
    cases, kjs = [], []
    for p in points:
        cases.append(synth.make_wake_case(p.case, nsteps=run_steps + 1, pitch_deg=p.pitch_deg))
        kjs.append(synth.make_kj_case(p.case, nsteps=run_steps + 1, pitch_deg=p.pitch_deg,
                                      root_cut=root_cut))
    return cases, kjs


def run(points, run_steps: int, relax=0.3, tol=1e-6, maxiter=100, mlp=None, precision="f32c",
        record=False, graph=True, root_cut: float = ROOT_CUT):
    """Runs every point for ``run_steps`` pcc steps with the lifting line.
    Returns per-step, per-case iterations, the lifting-line evaluations per
    step (the batch iterates until its slowest case converged), the bound
    circulation, rotor thrust and power after every step and, with
    ``record``, the training pairs."""
    cases, kjs = build(points, run_steps, root_cut)
    b = WakeBatch(cases, integrator="pcc", precision=precision)
    b.set_kj(kjs, relax=relax, tol=tol, maxiter=maxiter)
    if mlp is not None:
        b.set_mlp(mlp)
    n = len(points)
    lifting = [kj["foil"] == 0 for kj in kjs]  # stations with the lifting polar
    aoa_max = np.zeros(n)
    iters = np.zeros((run_steps, n), dtype=np.int64)
    evals = np.zeros(run_steps, dtype=np.int64)
    thrust = np.zeros((run_steps, n))
    power = np.zeros((run_steps, n))
    bounds = []
    X, dG, tag, lrows = [], [], [], []
    nbs = [c["nb"] for c in cases]
    aoa_prev = [np.zeros((c["nst"] - 1, c["nb"])) for c in cases]  # the engine's before step 0
    t0 = time.perf_counter()
    for s in range(run_steps):
        b.step(1, graph=graph)
        it, _, ev = b.kj_stats()
        iters[s] = it
        evals[s] = ev
        thrust[s], _, power[s] = b.loads()
        conv = [b.bound(k) for k in range(n)]
        aoas = [b.perf(k)[2] for k in range(n)]
        for k in range(n):
            aoa_max[k] = max(aoa_max[k], float(np.nanmax(np.abs(aoas[k][lifting[k]]))))
        if record:
            for k in range(n):
                if it[k] < maxiter:  # converged pairs only
                    x = b.kj_features(k)
                    X.append(x)
                    dG.append(conv[k].ravel(order="F") - x[:, 8].astype(np.float64))
                    tag.append(np.full((x.shape[0], 2), (s, k), dtype=np.int32))
                    lrows.append(start_rows(kjs[k], nbs[k], aoa_prev[k]))
        aoa_prev = aoas
        bounds.append(conv)
    wall = time.perf_counter() - t0
    b.close()
    out = dict(iters=iters, evals=evals, bounds=bounds, wall_s=wall, aoa_max=aoa_max,
               thrust=thrust, power=power)
    if record:
        out["X"] = np.concatenate(X).astype(np.float32) if X else np.zeros((0, N_FEATURES), np.float32)
        out["dG"] = np.concatenate(dG).astype(np.float32) if dG else np.zeros(0, np.float32)
        out["step_case"] = np.concatenate(tag) if tag else np.zeros((0, 2), np.int32)
        out["lift"] = np.concatenate(lrows) if lrows else np.zeros(0, bool)
    return out


def attached(points, run_steps=12, stall_deg=12.0, **kw):
    """The points whose plain solution keeps every lifting station below
    stall (|AoA| < stall_deg): there the fixed point is unique, so the start
    value changes iterations but not the converged circulation. (The
    synthetic polar drops from 1.28 to 0.49 at 12 deg; a station past it can
    have two fixed points, and any change of start value may select the
    other one.)"""
    r = run(points, run_steps, **kw)
    return [p for p, a in zip(points, r["aoa_max"]) if a < stall_deg]


def train(X, dG, epochs=30, batch=4096, lr=2e-3, seed=0, weight_decay=0.0, base="previous"):
    """An MLP fitted to dG (the change of the converged bound circulation
    over the previous step's) from the features X, with standardised inputs
    and target; Adam with the learning rate stepped down (x1, x1/4, x1/16)
    over three equal phases. ``base="extrapolated"``: the network learns the
    residual dG - dGamma_prev of the linear extrapolation (feature 9) and the
    wake engine adds its output to that extrapolation."""
    target = dG - X[:, 9] if base == "extrapolated" else dG
    shift = X.mean(0)
    sd = X.std(0)
    scale = np.where(sd > 0, 1.0 / np.maximum(sd, 1e-12), 1.0).astype(np.float32)
    out_scale = float(max(target.std(), 1e-12))
    m = Mlp(N_FEATURES, seed=seed)
    m.set_scaling(shift.astype(np.float32), scale, out_scale)
    m.set_base(base)
    losses = []
    per = [epochs - 2 * (epochs // 3), epochs // 3, epochs // 3]
    for k, (ep, f) in enumerate(zip(per, (1.0, 0.25, 0.0625))):
        if ep > 0:
            losses.append(m.train(X, target / out_scale, epochs=ep, batch=batch, lr=lr * f,
                                  seed=seed + 1 + k, weight_decay=weight_decay))
    m.shrink, m.full_out_scale = 1.0, out_scale
    return m, np.concatenate(losses) if losses else np.zeros(0)


def choose_shrink(m, points, run_steps, skip=4, alphas=(0.0, 0.25, 0.5, 0.75, 1.0), guard=1e-2,
                  guard_thrust=1e-3, **kw):
    """Scales the network's output by the alpha of ``alphas`` whose start
    value needs the fewest iterations (steps >= ``skip``, (step, case) pairs
    converged under the reference and every valid alpha) when the solver actually runs on
    ``points`` -- validation points kept out of the training pairs. The
    stopping rule sees the largest spanwise residual, and how fast the fixed
    point damps a start error depends on its spanwise shape, so no error
    norm of the start value predicts this as well as the iteration itself.
    alpha = 0 leaves the base alone.

    A candidate counts only if, at the last step, every case that reached
    its fixed point under the reference's previous-step start reaches one
    under the candidate too, and every case ends within ``guard`` (relative
    to its largest |Gamma| + 1) of the reference's bound circulation with
    its rotor thrust within ``guard_thrust`` (relative): past stall a station
    can have two fixed points and another start may select the other one
    (thrust percent apart, where starts on the same branch drift apart by a
    few 1e-4 over a run at tol 1e-6). Cases that stop at ``maxiter`` are
    compared too: comparing only the converged ones let a start through
    that moved a converged case of a later run to the other fixed point. If
    no candidate passes, the network falls back to the previous-step base
    with alpha = 0 (the reference's start). Sets
    ``m.shrink`` (and ``m.base``); ``m.validation`` lists (alpha, iterations,
    largest difference) per candidate."""
    shift, scale, _ = m.scaling()
    full = m.full_out_scale
    maxiter = kw.get("maxiter", 200)
    ref = run(points, run_steps, **kw)

    fixed = np.asarray(ref["iters"][-1]) < maxiter  # cases at a fixed point at the last step

    def largest_difference(r):
        return max(float(np.abs(np.asarray(x) - np.asarray(y)).max() / (np.abs(np.asarray(y)).max() + 1.0))
                   for x, y in zip(r["bounds"][-1], ref["bounds"][-1]))

    def thrust_difference(r):
        return float(np.max(np.abs(r["thrust"][-1] - ref["thrust"][-1]) / np.abs(ref["thrust"][-1])))

    its, valid, diffs = [], [], []
    for a in alphas:
        m.set_scaling(shift, scale, full * a)
        r = run(points, run_steps, mlp=m, **kw)
        its.append(r["iters"])
        diffs.append(largest_difference(r))
        keeps = bool(np.all(np.asarray(r["iters"][-1])[fixed] < maxiter))
        valid.append(keeps and diffs[-1] <= guard and thrust_difference(r) <= guard_thrust)
    ok = ref["iters"] < maxiter  # (step, case) pairs converged under the reference and every valid candidate
    for it, v in zip(its, valid):
        if v:
            ok &= it < maxiter
    ok[:skip] = False
    tot = [int(it[ok].sum()) if v else np.iinfo(np.int64).max for it, v in zip(its, valid)]
    m.validation = [(float(a), int(it[ok].sum()), d) for a, it, d in zip(alphas, its, diffs)]
    # iterations of the previous-step start over the same steps, and the chosen start's
    m.validation_reference = int(ref["iters"][ok].sum())
    if any(valid):
        k = int(np.argmin(tot))
        m.shrink = float(alphas[k])
        m.validation_chosen = tot[k]
    else:
        m.set_base("previous")
        m.shrink = 0.0
        m.validation_chosen = m.validation_reference
    m.set_scaling(shift, scale, full * m.shrink)
    return m.shrink


def fit_start_value(X, dG, val_points, val_steps, bases=("previous", "extrapolated"), epochs=40,
                    seed=0, **kw):
    """One network per base trained on the pairs (X, dG), each output scale
    chosen on ``val_points`` (``choose_shrink``, with its guards); keeps the
    network whose chosen start saves the most iterations against the
    previous-step start on those validation runs. Returns it with
    ``m.bases_tried`` = [(base trained, base kept after the guards, output
    scale, fraction of validation iterations saved)]."""
    best, tried = None, []
    for base in bases:
        m, _ = train(X, dG, epochs=epochs, base=base, seed=seed)
        choose_shrink(m, val_points, val_steps, **kw)
        saving = 1.0 - m.validation_chosen / max(m.validation_reference, 1)
        tried.append((base, m.base, m.shrink, saving))
        if best is None or saving > best[1]:
            if best is not None:
                best[0].close()
            best = (m, saving)
        else:
            m.close()
    best[0].bases_tried = tried
    return best[0]


def extrapolation_only():
    """A start value with no learned part: the linear extrapolation
    Gamma_prev + dGamma_prev (an output scale of zero on the extrapolated base)."""
    m = Mlp(N_FEATURES, seed=0)
    m.set_scaling(np.zeros(N_FEATURES, np.float32), np.ones(N_FEATURES, np.float32), 0.0)
    m.set_base("extrapolated")
    return m


def study(n_train: int = 400, n_test: int = 120, train_steps: int = 42, test_steps: int = 30,
          skip: int = 4, epochs: int = 60, relax: float = 0.3, tol: float = 1e-6,
          maxiter: int = 200, seed: int = 1, precision: str = "f32c", base: str = "extrapolated",
          weight_decay: float = 0.0, tight_points: int = 6, tight_steps: int = 10,
          tight_tol: float = 1e-10):
    """Trains the start value on the attached-flow points among ``n_train``
    seeded candidates (pairs from steps >= ``skip``, past the start-up
    transient of the synthetic initial circulation) and compares the
    iteration with and without it on the attached points among ``n_test``
    other candidates; also the extrapolation alone (no network), so the
    network's own share shows (``arms``: previous-step start, extrapolation
    alone, network, over the steps past the start-up that converged in all
    three). Converged results: thrust, power and bound circulation of each
    start against the previous-step start over the run at the study's
    tolerance (the stopping rule bounds the residual, not the distance to the
    fixed point, and each step's difference carries into the wake), and
    (``tight``) from one and the same wake state on ``tight_points`` test
    points at ``tight_tol`` in FP64, where every start must reach the same
    fixed point. Returns a dict of the measurements."""
    t0 = time.perf_counter()
    kw = dict(relax=relax, tol=tol, maxiter=maxiter, precision=precision)
    train_pts = attached(operating_points(n_train, seed=seed), **kw)
    d = run(train_pts, train_steps, record=True, **kw)
    keep = (d["step_case"][:, 0] >= skip) & d["lift"]
    t1 = time.perf_counter()
    # pairs from most points; the rest validate the network's output scale
    n_val = max(1, len(train_pts) // 5)
    fit_rows = keep & (d["step_case"][:, 1] < len(train_pts) - n_val)
    m, losses = train(d["X"][fit_rows], d["dG"][fit_rows], epochs=epochs, seed=seed, base=base,
                      weight_decay=weight_decay)
    choose_shrink(m, train_pts[-n_val:], test_steps, skip=skip, **kw)
    t2 = time.perf_counter()
    test_pts = attached(operating_points(n_test, seed=seed + 1), **kw)
    a = run(test_pts, test_steps, **kw)
    b = run(test_pts, test_steps, mlp=m, **kw)
    xo = extrapolation_only()
    e = run(test_pts, test_steps, mlp=xo, **kw)
    xo.close()
    ia, ib, ie = a["iters"], b["iters"], e["iters"]
    all3 = (ia < maxiter) & (ib < maxiter) & (ie < maxiter)
    all3[:skip] = False
    # iterations are compared over (step, case) that converged in both runs;
    # the converged circulation over cases that converged at every step
    both = (ia < maxiter) & (ib < maxiter)
    steady = both.copy()
    steady[:skip] = False
    ok_case = np.all(both, axis=0)
    rel = [float(np.abs(np.asarray(x) - np.asarray(y)).max() / (np.abs(np.asarray(x)).max() + 1.0))
           for k, (x, y) in enumerate(zip(a["bounds"][-1], b["bounds"][-1])) if ok_case[k]]
    ms, nsteps = m.train_stats()

    def loads_diff(x, y, mask):
        dT = np.abs(x["thrust"] - y["thrust"]) / np.abs(y["thrust"])
        dP = np.abs(x["power"] - y["power"]) / np.maximum(np.abs(y["power"]), 1e-9 * np.abs(y["thrust"]))
        return (float(dT[mask].max()) if mask.any() else 0.0,
                float(dP[mask].max()) if mask.any() else 0.0)

    def arm(r):
        return dict(iterations=int(r["iters"][all3].sum()), evals=int(r["evals"].sum()),
                    converged=float((r["iters"] < maxiter).mean()))

    arms = dict(previous=arm(a), extrapolated=arm(e), network=arm(b))
    for name, r in (("extrapolated", e), ("network", b)):
        arms[name]["thrust_rel_diff_max"], arms[name]["power_rel_diff_max"] = loads_diff(r, a, all3)
    # the same wake state, three starts, a tight tolerance: every start must
    # reach the same fixed point. Three identical FP64 batches (the FP32c
    # sums' rounding keeps the residual above ~1e-7) step `tight_steps` steps
    # from the previous-step start, then one more step from the previous step,
    # the extrapolation alone and the network.
    tight = {}
    if tight_points > 0 and test_pts:
        pts_t = test_pts[:tight_points]
        cases_t, kjs_t = build(pts_t, tight_steps + 1)
        maxit = max(maxiter, 600)
        bs = []
        for _ in range(3):
            bt = WakeBatch(cases_t, integrator="pcc", precision="f64")
            bt.set_kj(kjs_t, relax=relax, tol=tight_tol, maxiter=maxit)
            bs.append(bt)
        for _ in range(tight_steps):
            for bt in bs:
                bt.step(1, graph=True)
        same_state = all(np.array_equal(bs[0].bound(k), bt.bound(k)) for bt in bs[1:]
                         for k in range(len(pts_t)))
        xo2 = extrapolation_only()
        bs[1].set_mlp(xo2)
        bs[2].set_mlp(m)
        for bt in bs:
            bt.step(1, graph=True)
        its = [bt.kj_stats()[0] for bt in bs]
        ok = np.all([it < maxit for it in its], axis=0)
        G = [[bt.bound(k) for k in range(len(pts_t))] for bt in bs]
        L = [bt.loads() for bt in bs]
        tight = dict(tol=tight_tol, points=len(pts_t), step=tight_steps, same_state_before=bool(same_state),
                     converged=float(ok.mean()),
                     iterations={n: int(it[ok].sum()) for n, it in zip(("previous", "extrapolated",
                                                                          "network"), its)})
        for a_i, name in ((1, "extrapolated"), (2, "network")):
            dG = max(float(np.abs(G[a_i][k] - G[0][k]).max() / (np.abs(G[0][k]).max() + 1.0))
                     for k in range(len(pts_t)) if ok[k])
            dT = float((np.abs(L[a_i][0] - L[0][0]) / np.abs(L[0][0]))[ok].max())
            dP = float((np.abs(L[a_i][2] - L[0][2]) / np.abs(L[0][2]))[ok].max())
            tight[name] = dict(bound_rel_diff_max=dG, thrust_rel_diff_max=dT, power_rel_diff_max=dP)
        for bt in bs:
            bt.close()
        xo2.close()
    return dict(
        model=m, train_points=len(train_pts), test_points=len(test_pts), arms=arms, tight=tight,
        pairs=int(keep.sum()), loss_first=float(losses[0]), loss_last=float(losses[-1]),
        data_s=t1 - t0, train_s=t2 - t1, train_device_ms=ms, adam_steps=nsteps,
        iters_plain=int(ia[both].sum()), iters_mlp=int(ib[both].sum()),
        iters_plain_steady=int(ia[steady].sum()), iters_mlp_steady=int(ib[steady].sum()),
        evals_plain=int(a["evals"].sum()), evals_mlp=int(b["evals"].sum()),
        converged_plain=float((ia < maxiter).mean()), converged_mlp=float((ib < maxiter).mean()),
        saved=1.0 - ib[both].sum() / max(ia[both].sum(), 1),
        saved_steady=1.0 - ib[steady].sum() / max(ia[steady].sum(), 1),
        base=base, base_used=m.base, output_shrink=m.shrink, validation=m.validation,
        iters_extrap_steady=int(ie[all3].sum()),
        saved_extrap_steady=1.0 - ie[all3].sum() / max(ia[all3].sum(), 1),
        saved_vs_extrap_steady=1.0 - ib[all3].sum() / max(ie[all3].sum(), 1),
        cases_improved=int((np.where(both, ib, 0).sum(0) < np.where(both, ia, 0).sum(0)).sum()),
        cases_compared=int(ok_case.sum()),
        bound_rel_diff_max=max(rel) if rel else 0.0,
        bound_rel_diff_median=float(np.median(rel)) if rel else 0.0,
        wall_plain_s=a["wall_s"], wall_mlp_s=b["wall_s"])
