"""CPU restatement of the warm-start network (test infrastructure only).

The learned start of the converged emission solve is a tanh MLP
16 -> 64 -> 64 -> 64 -> 1 whose kernels (lipika_b200/csrc/lpk_mlp.cu) run
BF16 tensor-core tiles with FP32 accumulation. This module computes the same
forward pass, mean-squared-error loss and gradient in float64 numpy,
rounding to bfloat16 (round to nearest even) at exactly the points where
the kernels do: the inputs, W1, W2, W3, the first two hidden layers after
tanh (the next layer's operand and the weight-gradient operands), and the
three pre-activation gradients dZ3, dZ2 and dZ1 (the operands of the
weight-gradient tiles and of dH2 = dZ3 W3, dH1 = dZ2 W2). Biases, w4, the
third hidden layer, the tanh derivatives and every accumulation stay in
full precision.

It also restates the network's analytic feature layer (the circular orbit's
state from its elements, src/geometry/kepler.rs:32-85, and the 16
features) in float64.
"""
from __future__ import annotations

import numpy as np

N_F, N_H = 16, 64
OFF_W1 = 0
OFF_B1 = OFF_W1 + N_H * N_F
OFF_W2 = OFF_B1 + N_H
OFF_B2 = OFF_W2 + N_H * N_H
OFF_W3 = OFF_B2 + N_H
OFF_B3 = OFF_W3 + N_H * N_H
OFF_W4 = OFF_B3 + N_H
OFF_B4 = OFF_W4 + N_H
N_PARAMS = OFF_B4 + 1
TENSORS = (("W1", OFF_W1, OFF_B1), ("b1", OFF_B1, OFF_W2), ("W2", OFF_W2, OFF_B2), ("b2", OFF_B2, OFF_W3),
           ("W3", OFF_W3, OFF_B3), ("b3", OFF_B3, OFF_W4), ("w4", OFF_W4, OFF_B4), ("b4", OFF_B4, N_PARAMS))

GM = 3.986005e14                # src/geometry/kepler.rs:12
EARTH_RATE = 7.2921151467e-5    # src/channel/mod.rs:27
C = 299792458.0                 # src/lib.rs:53


def bf16(x):
    """Round float32 values to bfloat16 (nearest, ties to even); float64 out."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32)).view(np.uint32).astype(np.uint64)
    r = ((a + 0x7FFF + ((a >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return (p[OFF_W1:OFF_B1].reshape(N_H, N_F), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(N_H, N_H),
            p[OFF_B2:OFF_W3], p[OFF_W3:OFF_B3].reshape(N_H, N_H), p[OFF_B3:OFF_W4], p[OFF_W4:OFF_B4], p[OFF_B4])


def forward(p, x, quantize=True):
    q = bf16 if quantize else (lambda v: np.asarray(v, dtype=np.float64))
    w1, b1, w2, b2, w3, b3, w4, b4 = unpack(p)
    xq = q(x)
    h1 = np.tanh(xq @ q(w1).T + b1)
    h1q = q(h1)
    h2 = np.tanh(h1q @ q(w2).T + b2)
    h2q = q(h2)
    h3 = np.tanh(h2q @ q(w3).T + b3)
    y = h3 @ w4 + b4
    return y, (xq, h1, h1q, h2, h2q, h3)


def loss_grad(p, x, t, quantize=True):
    """Mean squared error and its gradient in the flat parameter layout."""
    q = bf16 if quantize else (lambda v: np.asarray(v, dtype=np.float64))
    w1, b1, w2, b2, w3, b3, w4, b4 = unpack(p)
    y, (xq, h1, h1q, h2, h2q, h3) = forward(p, x, quantize)
    n = len(x)
    e = y - np.asarray(t, dtype=np.float64)
    dy = 2.0 * e / n
    g = np.zeros(N_PARAMS)
    g[OFF_W4:OFF_B4] = h3.T @ dy
    g[OFF_B4] = dy.sum()
    dz3 = dy[:, None] * w4[None, :] * (1.0 - h3 * h3)
    g[OFF_B3:OFF_W4] = dz3.sum(0)
    dz3q = q(dz3)
    g[OFF_W3:OFF_B3] = (dz3q.T @ h2q).ravel()
    dz2 = (dz3q @ q(w3)) * (1.0 - h2 * h2)
    g[OFF_B2:OFF_W3] = dz2.sum(0)
    dz2q = q(dz2)
    g[OFF_W2:OFF_B2] = (dz2q.T @ h1q).ravel()
    dz1 = (dz2q @ q(w2)) * (1.0 - h1 * h1)
    g[OFF_B1:OFF_W2] = dz1.sum(0)
    g[OFF_W1:OFF_B1] = (q(dz1).T @ xq).ravel()
    return float(np.mean(e * e)), g


def orbit_state(orbit, e):
    """Position and velocity (ECEF) of a circular orbit (semi-major axis m,
    inclination, RAAN, true anomaly at epoch in degrees) e seconds after its
    epoch: CircularKeplerian::position_ecef's expression and its derivative."""
    a, inc, raan, ta = orbit
    e = np.asarray(e, dtype=np.float64)
    mm = np.sqrt(GM / (a * a * a))
    nu = np.radians(ta) + mm * e
    si, ci, so, co = np.sin(np.radians(inc)), np.cos(np.radians(inc)), np.sin(np.radians(raan)), np.cos(np.radians(raan))
    xp, yp = a * np.cos(nu), a * np.sin(nu)
    dxp, dyp = -a * mm * np.sin(nu), a * mm * np.cos(nu)
    y1, z1, dy1, dz1 = yp * ci, yp * si, dyp * ci, dyp * si
    xe, ye = xp * co - y1 * so, xp * so + y1 * co
    dxe, dye = dxp * co - dy1 * so, dxp * so + dy1 * co
    s, c = np.sin(EARTH_RATE * e), np.cos(EARTH_RATE * e)
    px, py = xe * c + ye * s, -xe * s + ye * c
    vx, vy = dxe * c + dye * s + EARTH_RATE * py, -dxe * s + dye * c - EARTH_RATE * px
    return np.stack([px, py, z1], -1), np.stack([vx, vy, dz1], -1)


def features(orbit, orbit_epoch, rx, epoch, t):
    """The 16 raw features of (orbit, receiver, reception times t) and the
    orbit's range R at each t."""
    t = np.asarray(t, dtype=np.float64)
    p, v = orbit_state(orbit, (epoch - orbit_epoch) + t)
    d = p - np.asarray(rx)[None, :]
    R = np.linalg.norm(d, axis=1)
    u = d / R[:, None]
    f = np.zeros((len(t), N_F))
    f[:, 0:4] = np.asarray(orbit)[None, :]
    f[:, 4:7] = np.asarray(rx)[None, :]
    f[:, 7] = t
    f[:, 8:11] = u
    f[:, 11] = R / C
    f[:, 12] = np.sum(v * u, axis=1) / C
    f[:, 13] = v[:, 0] / C
    f[:, 14] = v[:, 1] / C
    f[:, 15] = EARTH_RATE * (p[:, 0] * rx[1] - p[:, 1] * rx[0]) / R / C
    return f, R
