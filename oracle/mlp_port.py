"""CPU restatement of the VCA surrogate network (pyqcm_b200/csrc/mlp.cu) for
checking its GPU forward pass and gradients.

TEST INFRASTRUCTURE ONLY -- imported by tests/, never by the product package.
There is no counterpart in the reference: the network is this project's own.
The same rounding points as the GPU: inputs, weights, hidden activations and
the back-propagated pre-activation gradients rounded to BF16 (round to nearest
even) before each matrix product; products, sums and the head in FP32 or
better (float64 here)."""
from __future__ import annotations

import numpy as np
from math import erf, sqrt, pi, exp

_erf = np.vectorize(erf)


def bf16(x):
    """Round float32 values to the nearest BF16 (ties to even), returned as float32."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + _erf(z / sqrt(2.0))) + z * np.exp(-0.5 * z * z) / sqrt(2.0 * pi)


def forward(blocks, x, n_in):
    W1, b1, W2, b2, W3, b3, w4, b4 = [np.asarray(b, dtype=np.float64) for b in blocks]
    k_in = W1.shape[1]
    X = np.zeros((len(x), k_in))
    X[:, :n_in] = bf16(np.asarray(x, dtype=np.float32))
    cache = {"X": X}
    h = X
    for l, (W, b) in enumerate(((W1, b1), (W2, b2), (W3, b3))):
        z = h @ bf16(W.astype(np.float32)).astype(np.float64).T + b
        z = z.astype(np.float32).astype(np.float64)
        h = bf16(gelu(z).astype(np.float32)).astype(np.float64)
        cache[f"Z{l}"] = z
        cache[f"H{l}"] = h
    y = h @ bf16(w4.astype(np.float32)).astype(np.float64) + b4[0]
    return y, cache


def gradients(blocks, x, t, n_in):
    """MSE loss and the gradient blocks (dW1, db1, dW2, db2, dW3, db3, dw4, db4)."""
    W1, b1, W2, b2, W3, b3, w4, b4 = [np.asarray(b, dtype=np.float64) for b in blocks]
    y, c = forward(blocks, x, n_in)
    n = len(x)
    d = y - np.asarray(t, dtype=np.float64)
    loss = float(np.sum(d * d) / n)
    dy = 2.0 * d / n
    g = [None] * 8
    g[6] = dy @ c["H2"]
    g[7] = np.array([dy.sum()])
    w4h = bf16(w4.astype(np.float32)).astype(np.float64)
    dz = np.outer(dy, w4h) * gelu_grad(c["Z2"])
    Ws = [W1, W2, W3]
    for l in (2, 1, 0):
        dzh = bf16(dz.astype(np.float32)).astype(np.float64)
        prev = c[f"H{l - 1}"] if l > 0 else c["X"]
        g[2 * l] = dzh.T @ prev
        g[2 * l + 1] = dz.sum(axis=0)
        if l > 0:
            dh = dzh @ bf16(Ws[l].astype(np.float32)).astype(np.float64)
            dz = dh * gelu_grad(c[f"Z{l - 1}"])
    return loss, g
