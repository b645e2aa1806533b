"""CPU tests of the start value's output-scale selection
(gamma_init.choose_shrink) with the solver runs replaced by a fake: the
fewest-iterations choice, the fixed-point guard and the fallback to the
reference's previous-step start."""
from __future__ import annotations

import importlib

import numpy as np


class FakeMlp:
    def __init__(self, base="extrapolated"):
        self.base, self.full_out_scale, self.out = base, 2.0, 2.0

    def scaling(self):
        return np.zeros(11, np.float32), np.ones(11, np.float32), self.out

    def set_scaling(self, shift, scale, out_scale):
        self.out = out_scale

    def set_base(self, base):
        self.base = base


def _fake_run(table):
    """run() stand-in: iterations and final bounds by the network's output
    scale (None: the reference's previous-step start)."""
    def run(points, steps, mlp=None, **kw):
        key = None if mlp is None else round(mlp.out / mlp.full_out_scale, 2)
        its, bound = table[key][:2]
        thrust = table[key][2] if len(table[key]) > 2 else 1.0
        return {"iters": np.array(its), "bounds": [[np.array(bound)]],
                "thrust": np.array([[thrust]])}
    return run


def test_choose_shrink_takes_the_fewest_iterations(monkeypatch):
    gi = importlib.import_module("winds-master_b200.gamma_init")
    ref = [10.0, 20.0]
    table = {None: ([[9], [9], [9], [9], [9], [40]], ref)}
    for a, it in zip((0.0, 0.25, 0.5, 0.75, 1.0), (30, 20, 25, 35, 50)):
        table[a] = ([[9], [9], [9], [9], [9], [it]], [10.0 + 1e-5, 20.0])
    monkeypatch.setattr(gi, "run", _fake_run(table))
    m = FakeMlp()
    assert gi.choose_shrink(m, [], 6, skip=4) == 0.25
    assert m.out == 0.5 and m.base == "extrapolated"
    assert [v[1] for v in m.validation] == [39, 29, 34, 44, 59]  # steps 4 and 5


def test_choose_shrink_rejects_another_fixed_point(monkeypatch):
    gi = importlib.import_module("winds-master_b200.gamma_init")
    ref = [10.0, 20.0]
    table = {None: ([[9], [9], [9], [9], [9], [40]], ref)}
    for a, it, b in zip((0.0, 0.25, 0.5, 0.75, 1.0), (30, 20, 25, 35, 50),
                        (ref, [12.0, 20.0], ref, ref, ref)):
        table[a] = ([[9], [9], [9], [9], [9], [it]], b)
    monkeypatch.setattr(gi, "run", _fake_run(table))
    m = FakeMlp()
    # 0.25 is fastest but lands elsewhere (2/21 > 1e-2): the next best valid is 0.5
    assert gi.choose_shrink(m, [], 6, skip=4) == 0.5


def test_choose_shrink_falls_back_to_the_reference_start(monkeypatch):
    gi = importlib.import_module("winds-master_b200.gamma_init")
    ref = [10.0, 20.0]
    table = {None: ([[9], [9], [9], [9], [9], [40]], ref)}
    for a in (0.0, 0.25, 0.5, 0.75, 1.0):
        table[a] = ([[9], [9], [9], [9], [9], [20]], [14.0, 20.0])
    monkeypatch.setattr(gi, "run", _fake_run(table))
    m = FakeMlp()
    assert gi.choose_shrink(m, [], 6, skip=4) == 0.0
    assert m.base == "previous" and m.out == 0.0


def test_start_rows_follow_the_stall_bounds():
    """The synthetic polar's highest Cl in [0, 45] deg is at its 12 deg stall
    (and the lowest in [-45, 0] at -12 deg); the start value applies at
    lifting stations whose last AoA is more than 2 deg inside those bounds."""
    gi = importlib.import_module("winds-master_b200.gamma_init")
    synth = importlib.import_module("winds-master_b200.synth")
    rc = synth.RotorCase(nst=9, nsteps=4, seed=1)
    kj = synth.make_kj_case(rc, nsteps=4, root_cut=0.2)
    sb = gi.stall_bounds(kj)
    lift = gi.lifting_stations(kj)
    assert lift.any() and not lift.all()
    np.testing.assert_allclose(sb[lift], np.tile([-12.0, 12.0], (lift.sum(), 1)), atol=0.3)
    ns, nb = len(lift), rc.nb
    aoa = np.zeros((ns, nb))
    aoa[:, 1] = 11.0  # past stall less the margin on blade 1
    aoa[:, 2] = -9.0
    rows = gi.start_rows(kj, nb, aoa).reshape(ns, nb, order="F")
    np.testing.assert_array_equal(rows[:, 0], lift)
    assert not rows[:, 1].any()
    np.testing.assert_array_equal(rows[:, 2], lift)


def test_choose_shrink_rejects_a_thrust_jump(monkeypatch):
    """Circulation within the guard but thrust 2% off the previous-step
    start's: another fixed point, rejected."""
    gi = importlib.import_module("winds-master_b200.gamma_init")
    ref = [10.0, 20.0]
    table = {None: ([[9], [9], [9], [9], [9], [40]], ref, 1.0)}
    for a, it, t in zip((0.0, 0.25, 0.5, 0.75, 1.0), (30, 20, 25, 35, 50),
                        (1.0, 1.02, 1.0001, 1.0, 1.0)):
        table[a] = ([[9], [9], [9], [9], [9], [it]], ref, t)
    monkeypatch.setattr(gi, "run", _fake_run(table))
    m = FakeMlp()
    assert gi.choose_shrink(m, [], 6, skip=4) == 0.5


def test_fit_start_value_keeps_the_base_that_saves_more(monkeypatch):
    """One network per base; the one whose chosen output scale saves more
    validation iterations is kept, the other is closed."""
    gi = importlib.import_module("winds-master_b200.gamma_init")
    closed = []

    class Net(FakeMlp):
        def close(self):
            closed.append(self.base)

    def train(X, dG, epochs=30, base="previous", seed=0, **kw):
        return Net(base), None

    def choose_shrink(m, points, steps, **kw):
        m.validation_reference = 100
        m.validation_chosen = {"previous": 90, "extrapolated": 80}[m.base]
        m.shrink = 0.5
        return m.shrink

    monkeypatch.setattr(gi, "train", train)
    monkeypatch.setattr(gi, "choose_shrink", choose_shrink)
    m = gi.fit_start_value(None, None, [], 6)
    assert m.base == "extrapolated" and closed == ["previous"]
    assert [(b, round(s, 6)) for b, _, _, s in m.bases_tried] == [("previous", 0.1),
                                                                   ("extrapolated", 0.2)]


def test_choose_shrink_keeps_convergence(monkeypatch):
    """A candidate that leaves a case the reference start converged at
    maxiter is rejected, and the iterations are compared over the pairs that
    converged under the reference and every valid candidate."""
    gi = importlib.import_module("winds-master_b200.gamma_init")

    def run(points, steps, mlp=None, **kw):
        key = None if mlp is None else round(mlp.out / mlp.full_out_scale, 2)
        last = {None: [40, 40], 0.0: [30, 40], 0.25: [200, 20], 0.5: [25, 40], 0.75: [35, 40],
                1.0: [50, 40]}[key]
        return {"iters": np.array([[9, 9]] * 5 + [last]), "bounds": [[np.array([10.0, 20.0])] * 2],
                "thrust": np.array([[1.0, 1.0]])}

    monkeypatch.setattr(gi, "run", run)
    m = FakeMlp()
    # 0.25 is fastest on case 1 but leaves case 0 at maxiter: the next best valid is 0.5
    assert gi.choose_shrink(m, [], 6, skip=4) == 0.5
    assert [v[1] for v in m.validation][2] == 18 + 25 + 40
