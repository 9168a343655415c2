"""A float64 NumPy restatement of the surrogate network's forward and backward pass, used by the
tests as the CPU checker of the GPU kernels' gradients (test infrastructure).

It reproduces the GPU's storage precisions at the same points — BF16 inputs, weights, hidden
activations and output gradients; FP32 pre-activations — so that the remaining difference is only
the order of the FP32 accumulations and the hardware tanh's approximation (about 2^-11
relative)."""

from __future__ import annotations

import math

import numpy as np


def bf16(x: np.ndarray) -> np.ndarray:
    """Round to bfloat16 (round to nearest even on the upper 16 bits of float32), as float64."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    r = ((u + 0x7FFF + lsb) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


K0, K1 = math.sqrt(2.0 / math.pi), 0.044715  # GELU in its tanh form, as the kernels compute it


def gelu(x):
    return 0.5 * x * (1.0 + np.tanh(K0 * (x + K1 * x ** 3)))


def gelu_grad(x):
    t = np.tanh(K0 * (x + K1 * x ** 3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * K0 * (1.0 + 3.0 * K1 * x * x)


def forward_backward(X, Ws, bs, Y, n_out: int, scale: float):
    """X: (B, K0) bf16 values; Ws[l]: (n_l, k_l) bf16 values; bs[l]: (n_l,); Y: (B, n_out).
    Returns (loss, gW list, gb list, pred)."""
    L = len(Ws)
    Z, H = [], []
    h = X
    for li in range(L):
        z = h @ Ws[li].T + bs[li]
        Z.append(z)
        if li < L - 1:
            h = bf16(gelu(z))
            H.append(h)
    pred = Z[-1]
    d = np.zeros_like(pred)
    d[:, :n_out] = pred[:, :n_out] - Y
    loss = scale * float((d ** 2).sum())
    dZ = bf16(2.0 * scale * d)
    gW, gb = [None] * L, [None] * L
    for li in range(L - 1, -1, -1):
        prev = X if li == 0 else H[li - 1]
        gW[li] = dZ.T @ prev
        gb[li] = dZ.sum(0)
        if li > 0:
            dZ = bf16((dZ @ Ws[li]) * gelu_grad(Z[li - 1]))
    return loss, gW, gb, pred
