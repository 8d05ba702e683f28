"""CPU restatement of the learned-placement network (test infrastructure:
imported only by tests/).

Follows the GPU kernels of gpu_cdt_refine_b200/csrc/learned.cu and
learned.cuh step by step: inputs, weights and activations rounded to bf16 at
the same points (round to nearest even), sums in float64 (the GPU sums in
fp32 on the tensor cores, so the comparison allows for rounding order), ReLU
derivative taken where the bf16 activation is non-zero, loss the mean squared
error.  Parameter layout: W1[64][32], b1[64], W2[64][64], b2[64], w3[64], b3.
"""
from __future__ import annotations

import numpy as np

F, H = 32, 64
OFF_W1 = 0
OFF_B1 = OFF_W1 + H * F
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + H
NPARAM = OFF_B3 + 1


_ROUND = [True]


def bf16(x):
    """Round float32 values to bfloat16 (nearest even), returned as float64
    (no rounding inside `exact_arithmetic()`)."""
    if not _ROUND[0]:
        return np.asarray(x, np.float64)
    a = np.ascontiguousarray(np.asarray(x, np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


class exact_arithmetic:
    """Context in which the restatement runs in float64 without bf16 rounding,
    to check its backward pass against finite differences."""

    def __enter__(self):
        _ROUND[0] = False

    def __exit__(self, *a):
        _ROUND[0] = True


def unpack(p):
    p = np.asarray(p, np.float32 if _ROUND[0] else np.float64)
    return (p[OFF_W1:OFF_B1].reshape(H, F), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(H, H), p[OFF_B2:OFF_W3],
            p[OFF_W3:OFF_B3], p[OFF_B3])


def forward(p, X):
    W1, b1, W2, b2, w3, b3 = unpack(p)
    ft = np.float32 if _ROUND[0] else np.float64
    x = bf16(X)
    z1 = (x @ bf16(W1).T).astype(ft) + b1
    a1 = bf16(np.maximum(z1, 0))
    z2 = (a1 @ bf16(W2).T).astype(ft) + b2
    a2 = bf16(np.maximum(z2, 0))
    y = a2 @ bf16(w3) + np.float64(b3)
    return x, a1, a2, y


def loss_and_grad(p, X, T):
    """Mean squared error and its gradient, restated from k_mlp_fwd_bwd."""
    W1, b1, W2, b2, w3, b3 = unpack(p)
    n = X.shape[0]
    x, a1, a2, y = forward(p, X)
    ft = np.float32 if _ROUND[0] else np.float64
    err = (y - np.asarray(T, np.float64)).astype(ft)
    loss = float(np.sum(err.astype(np.float64) ** 2) / n)
    dy = (2.0 * err / n).astype(ft)
    g = np.zeros(NPARAM, np.float64)
    g[OFF_W3:OFF_B3] = dy @ a2
    g[OFF_B3] = dy.sum()
    dz2 = bf16(np.where(a2 != 0, dy[:, None].astype(np.float64) * bf16(w3)[None, :], 0.0))
    g[OFF_W2:OFF_B2] = (dz2.T @ a1).ravel()
    g[OFF_B2:OFF_W3] = dz2.sum(0)
    dh1 = (dz2 @ bf16(W2)).astype(ft)
    dz1 = bf16(np.where(a1 != 0, dh1, 0.0))
    g[OFF_W1:OFF_B1] = (dz1.T @ x).ravel()
    g[OFF_B1:OFF_W2] = dz1.sum(0)
    return loss, g
