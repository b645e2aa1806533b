"""GPU tests of the MLP kernels (include/winds_mlp.h): forward and the full
parameter gradient of the tcgen05 BF16 GEMM path against the NumPy oracle
(oracle/mlp_ref.py), deterministic reductions, and Adam training."""
from __future__ import annotations

import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _model(n_in=9, seed=5):
    mlp = importlib.import_module("winds-master_b200.mlp")
    return mlp.Mlp(n_in, seed=seed)


def _data(n, n_in=9, seed=0):
    rng = np.random.default_rng(seed)
    x = rng.normal(0, 1, (n, n_in)).astype(np.float32) * 2.0 + 0.5
    t = (np.sin(x[:, 0]) + 0.3 * x[:, 1] * x[:, 2] - 0.2 * x[:, 3] ** 2).astype(np.float32)
    return x, t


def _blocks(mlp_ref):
    out = []
    for L in range(4):
        out.append((f"W{L+1}", mlp_ref.OFF_W[L], mlp_ref.OFF_W[L] + 128 * mlp_ref.IN_K[L]))
        out.append((f"b{L+1}", mlp_ref.OFF_B[L], mlp_ref.OFF_B[L] + 128))
    out += [("w5", mlp_ref.OFF_W5, mlp_ref.OFF_W5 + 128), ("b5", mlp_ref.OFF_B5, mlp_ref.OFF_B5 + 1)]
    return out


@pytest.mark.parametrize("n", [1, 77, 300, 1024])
def test_forward_matches_oracle(wb, n):
    import mlp_ref
    m = _model()
    x, _ = _data(n)
    sh = np.full(9, 0.5, np.float32)
    sc = np.full(9, 0.5, np.float32)
    m.set_scaling(sh, sc, 1.0)
    y = m.forward(x)
    y16, _ = mlp_ref.forward(m.params, x, sh, sc, bf16_round=True)
    y64, _ = mlp_ref.forward(m.params, x, sh, sc)
    scale = np.abs(y64).max() + 1e-3
    assert np.abs(y - y16).max() <= 2e-3 * scale
    assert np.abs(y - y64).max() <= 3e-2 * scale
    m.close()


@pytest.mark.parametrize("n", [64, 333, 2048])
def test_gradient_matches_oracle(wb, n):
    """Every parameter block of the device gradient against the oracle with
    the same BF16 rounding points (tight) and in plain FP64 (loose)."""
    import mlp_ref
    m = _model(seed=11)
    x, t = _data(n, seed=2)
    sh = np.zeros(9, np.float32)
    sc = np.full(9, 0.5, np.float32)
    m.set_scaling(sh, sc, 1.0)
    loss, g = m.loss_grad(x, t)
    th = m.params
    l16, g16 = mlp_ref.loss_grad(th, x, t, sh, sc, bf16_round=True)
    l64, g64 = mlp_ref.loss_grad(th, x, t, sh, sc)
    assert abs(loss - l16) <= 1e-4 * l16
    assert abs(loss - l64) <= 2e-2 * l64
    for name, a, b in _blocks(mlp_ref):
        ref16, ref64, got = g16[a:b], g64[a:b], g[a:b]
        n16 = np.linalg.norm(ref16)
        assert np.linalg.norm(got - ref16) <= 5e-3 * n16 + 1e-7, (name, np.linalg.norm(got - ref16), n16)
        assert np.linalg.norm(got - ref64) <= 6e-2 * np.linalg.norm(ref64) + 1e-7, name
    # padded input columns of W1 carry no gradient
    W1 = g[mlp_ref.OFF_W[0]:mlp_ref.OFF_B[0]].reshape(128, 16)
    assert np.all(W1[:, 9:] == 0.0)
    m.close()


def test_gradient_is_deterministic(wb):
    m = _model(seed=3)
    x, t = _data(5000, seed=4)
    _, g1 = m.loss_grad(x, t)
    _, g2 = m.loss_grad(x, t)
    np.testing.assert_array_equal(g1, g2)
    m.close()


def test_training_reduces_loss_and_generalises(wb):
    m = _model(seed=7)
    x, t = _data(60000, seed=8)
    xv, tv = _data(4000, seed=9)
    sh = x.mean(0)
    sc = 1.0 / x.std(0)
    m.set_scaling(sh, sc, 1.0)
    l0 = 0.5 * float(np.mean((m.forward(xv) - tv) ** 2))
    el = m.train(x, t, epochs=8, batch=2048, lr=2e-3, seed=1)
    assert np.all(np.isfinite(el))
    assert el[-1] < 0.2 * el[0]
    lv = 0.5 * float(np.mean((m.forward(xv) - tv) ** 2))
    assert lv < 0.05 * l0, (l0, lv)
    ms, steps = m.train_stats()
    assert steps == 8 * ((60000 + 2047) // 2048) and ms > 0
    m.close()
