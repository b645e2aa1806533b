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
        its, bound = table[key]
        return {"iters": np.array(its), "bounds": [[np.array(bound)]]}
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
