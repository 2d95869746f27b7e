"""CPU restatement of the warm-start network (test infrastructure only).

The learned start of the converged emission solve is a tanh MLP
8 -> 64 -> 64 -> 1 whose kernels (lipika_b200/csrc/lpk_mlp.cu) run BF16
tensor-core tiles with FP32 accumulation. This module computes the same
forward pass, mean-squared-error loss and gradient in float64 numpy,
rounding to bfloat16 (round to nearest even) at exactly the points where
the kernels do: the inputs, W1, W2, the first hidden layer after tanh (the
second layer's operand), and the two pre-activation gradients dZ2 and dZ1
(the operands of the weight-gradient tiles and of dH1 = dZ2 W2). Biases,
w3, the second hidden layer and every accumulation stay in full precision.
"""
from __future__ import annotations

import numpy as np

N_F, N_H = 8, 64
OFF_W1 = 0
OFF_B1 = OFF_W1 + N_H * N_F
OFF_W2 = OFF_B1 + N_H
OFF_B2 = OFF_W2 + N_H * N_H
OFF_W3 = OFF_B2 + N_H
OFF_B3 = OFF_W3 + N_H
N_PARAMS = OFF_B3 + 1


def bf16(x):
    """Round float32 values to bfloat16 (nearest, ties to even); float64 out."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32)).view(np.uint32).astype(np.uint64)
    r = ((a + 0x7FFF + ((a >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return (p[OFF_W1:OFF_B1].reshape(N_H, N_F), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(N_H, N_H),
            p[OFF_B2:OFF_W3], p[OFF_W3:OFF_B3], p[OFF_B3])


def forward(p, x, quantize=True):
    q = bf16 if quantize else (lambda v: np.asarray(v, dtype=np.float64))
    w1, b1, w2, b2, w3, b3 = unpack(p)
    xq = q(x)
    h1 = np.tanh(xq @ q(w1).T + b1)
    h1q = q(h1)
    h2 = np.tanh(h1q @ q(w2).T + b2)
    y = h2 @ w3 + b3
    return y, (xq, h1, h1q, h2)


def loss_grad(p, x, t, quantize=True):
    """Mean squared error and its gradient in the flat parameter layout."""
    q = bf16 if quantize else (lambda v: np.asarray(v, dtype=np.float64))
    w1, b1, w2, b2, w3, b3 = unpack(p)
    y, (xq, h1, h1q, h2) = forward(p, x, quantize)
    n = len(x)
    e = y - np.asarray(t, dtype=np.float64)
    dy = 2.0 * e / n
    g = np.zeros(N_PARAMS)
    g[OFF_W3:OFF_B3] = h2.T @ dy
    g[OFF_B3] = dy.sum()
    dz2 = dy[:, None] * w3[None, :] * (1.0 - h2 * h2)
    g[OFF_B2:OFF_W3] = dz2.sum(0)
    dz2q = q(dz2)
    g[OFF_W2:OFF_B2] = (dz2q.T @ h1q).ravel()
    dz1 = (dz2q @ q(w2)) * (1.0 - h1 * h1)
    g[OFF_B1:OFF_W2] = dz1.sum(0)
    g[OFF_W1:OFF_B1] = (q(dz1).T @ xq).ravel()
    return float(np.mean(e * e)), g
