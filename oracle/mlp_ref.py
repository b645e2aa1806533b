"""NumPy oracle of the bound-circulation MLP (test infrastructure).

The network of ``include/winds_mlp.h``: inputs standardised as
``(x - shift) * scale`` and zero-padded to 16, four hidden layers of width
128 with GELU in its tanh form, a linear output; loss ``0.5 * mean((y-t)^2)``.
Parameters share the library's flat layout (``W1 [128][16], b1, W2 [128][128],
b2, W3, b3, W4, b4, w5 [128], b5``).

``bf16=False`` evaluates everything in FP64 (the mathematical reference, its
gradient pinned by finite differences in the tests). ``bf16=True`` rounds
where the device kernels round -- the standardised inputs, the weights, every
hidden activation and every back-propagated pre-activation gradient that
feeds a GEMM -- and keeps FP64 elsewhere, so the device result differs from
it only by FP32 accumulation order and math-library ulps.
"""
from __future__ import annotations

import numpy as np

WIDTH = 128
IN_PAD = 16
OFF_W = (0, 2176, 18688, 35200)
OFF_B = (2048, 18560, 35072, 51584)
OFF_W5 = 51712
OFF_B5 = 51840
N_PARAM = 51841
IN_K = (IN_PAD, WIDTH, WIDTH, WIDTH)
GELU_C = 0.7978845608028654
GELU_A = 0.044715


def bf16(x):
    """Round to the nearest BF16 (ties to even), returned as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).reshape(a.shape)


def gelu(z):
    return 0.5 * z * (1.0 + np.tanh(GELU_C * (z + GELU_A * z ** 3)))


def gelu_grad(z):
    t = np.tanh(GELU_C * (z + GELU_A * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * GELU_C * (1.0 + 3.0 * GELU_A * z * z)


def unpack(theta):
    th = np.asarray(theta, dtype=np.float64)
    Ws = [th[OFF_W[L]:OFF_W[L] + WIDTH * IN_K[L]].reshape(WIDTH, IN_K[L]) for L in range(4)]
    bs = [th[OFF_B[L]:OFF_B[L] + WIDTH] for L in range(4)]
    return Ws, bs, th[OFF_W5:OFF_W5 + WIDTH], th[OFF_B5]


def standardise(x, shift, scale, n_in, rnd):
    xs = np.zeros((np.shape(x)[0], IN_PAD), dtype=np.float64)
    if rnd:  # FP32 arithmetic, then BF16, as the device's input kernel
        x = np.asarray(x, dtype=np.float32)
        v = (x - np.asarray(shift[:n_in], np.float32)) * np.asarray(scale[:n_in], np.float32)
        xs[:, :n_in] = bf16(v)
    else:
        xs[:, :n_in] = (np.asarray(x, np.float64) - np.asarray(shift[:n_in], np.float64)) * \
            np.asarray(scale[:n_in], np.float64)
    return xs


def forward(theta, x, shift, scale, bf16_round=False):
    """Returns (y, cache) for rows x [n][n_in]."""
    n_in = x.shape[1]
    Ws, bs, w5, b5 = unpack(theta)
    r = (lambda a: bf16(a).astype(np.float64)) if bf16_round else (lambda a: a)
    f = (lambda a: np.float32(a).astype(np.float64)) if bf16_round else (lambda a: a)
    a = standardise(x, shift, scale, n_in, bf16_round)
    acts, zs = [a], []
    for L in range(4):
        z = acts[-1] @ r(Ws[L]).T + f(bs[L])
        if bf16_round:
            z = z.astype(np.float32).astype(np.float64)
        zs.append(z)
        acts.append(r(gelu(z)))
    y = acts[-1] @ f(w5) + float(f(b5))
    return y, dict(acts=acts, zs=zs, Ws=Ws, w5=w5, rnd=bf16_round)


def loss_grad(theta, x, t, shift, scale, bf16_round=False):
    """0.5 * mean((y - t)^2) and its gradient in the flat parameter layout."""
    y, c = forward(theta, x, shift, scale, bf16_round)
    n = x.shape[0]
    r = (lambda a: bf16(a).astype(np.float64)) if bf16_round else (lambda a: a)
    e = y - np.asarray(t, np.float64)
    loss = 0.5 * float(np.mean(e * e))
    dy = e / n
    g = np.zeros(N_PARAM)
    g[OFF_W5:OFF_W5 + WIDTH] = dy @ c["acts"][4]
    g[OFF_B5] = dy.sum()
    dz = dy[:, None] * c["w5"][None, :] * gelu_grad(c["zs"][3])
    for L in range(3, -1, -1):
        g[OFF_B[L]:OFF_B[L] + WIDTH] = dz.sum(0)
        dzr = r(dz)
        g[OFF_W[L]:OFF_W[L] + WIDTH * IN_K[L]] = (dzr.T @ c["acts"][L]).ravel()
        if L > 0:
            dz = (dzr @ r(c["Ws"][L])) * gelu_grad(c["zs"][L - 1])
    return loss, g
