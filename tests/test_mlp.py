"""CPU tests of the MLP oracle (oracle/mlp_ref.py): its FP64 gradient against
central finite differences, and the BF16 rounding it emulates."""
from __future__ import annotations

import numpy as np


def _setup(seed=0, n=48, n_in=9):
    import mlp_ref
    rng = np.random.default_rng(seed)
    th = np.zeros(mlp_ref.N_PARAM)
    for L in range(4):
        fan = n_in if L == 0 else mlp_ref.WIDTH
        W = rng.normal(0, 1 / np.sqrt(fan), (mlp_ref.WIDTH, mlp_ref.IN_K[L]))
        W[:, fan:] = 0.0
        th[mlp_ref.OFF_W[L]:mlp_ref.OFF_W[L] + W.size] = W.ravel()
        th[mlp_ref.OFF_B[L]:mlp_ref.OFF_B[L] + mlp_ref.WIDTH] = rng.normal(0, 0.1, mlp_ref.WIDTH)
    th[mlp_ref.OFF_W5:mlp_ref.OFF_W5 + mlp_ref.WIDTH] = rng.normal(0, 1 / np.sqrt(128), 128)
    th[mlp_ref.OFF_B5] = 0.05
    x = rng.normal(0, 1, (n, n_in))
    t = rng.normal(0, 1, n)
    return mlp_ref, th, x, t, np.zeros(n_in), np.ones(n_in)


def test_mlp_oracle_gradient_matches_finite_differences():
    mlp_ref, th, x, t, sh, sc = _setup()
    _, g = mlp_ref.loss_grad(th, x, t, sh, sc)
    rng = np.random.default_rng(1)
    # a sample of coordinates from every parameter block
    idx = []
    for L in range(4):
        idx += list(mlp_ref.OFF_W[L] + rng.integers(0, mlp_ref.WIDTH * (9 if L == 0 else 128), 6))
        idx += list(mlp_ref.OFF_B[L] + rng.integers(0, 128, 3))
    idx += list(mlp_ref.OFF_W5 + rng.integers(0, 128, 4)) + [mlp_ref.OFF_B5]
    h = 1e-6
    for i in idx:
        if mlp_ref.OFF_W[0] <= i < mlp_ref.OFF_B[0] and (i - mlp_ref.OFF_W[0]) % 16 >= 9:
            continue
        tp, tm = th.copy(), th.copy()
        tp[i] += h
        tm[i] -= h
        fd = (mlp_ref.loss_grad(tp, x, t, sh, sc)[0] - mlp_ref.loss_grad(tm, x, t, sh, sc)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, g[i])


def test_bf16_rounding_is_round_to_nearest_even():
    import mlp_ref
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 2 ** -9, 1.0 + 3 * 2 ** -9, -2.5, 3.0e38], np.float32)
    r = mlp_ref.bf16(x)
    assert r[0] == 1.0
    # 1 + 2^-8 is exactly halfway between BF16 neighbours 1 and 1 + 2^-7: ties to even -> 1
    assert r[1] == 1.0
    assert r[2] == 1.0
    assert r[3] == np.float32(1.0 + 2 ** -7)
    assert r[4] == -2.5
    # every rounded value has a zero low half
    assert np.all((r.view(np.uint32) & 0xFFFF) == 0)


def test_bf16_emulation_stays_close_to_fp64():
    mlp_ref, th, x, t, sh, sc = _setup(seed=3)
    l64, g64 = mlp_ref.loss_grad(th, x, t, sh, sc)
    l16, g16 = mlp_ref.loss_grad(th, x, t, sh, sc, bf16_round=True)
    assert abs(l16 - l64) <= 2e-2 * l64
    assert np.linalg.norm(g16 - g64) <= 5e-2 * np.linalg.norm(g64)
