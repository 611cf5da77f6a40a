"""CPU oracle of the learned-MAC network.  TEST INFRASTRUCTURE ONLY.

The 8-64-64-1 MLP with ReLU has no counterpart in the reference; this numpy
restatement is the checker of the engine's tensor-core forward/backward
kernels.  `bf16=True` rounds to BF16 at exactly the points where the kernels
do (normalised inputs, W1, W2, the hidden activation h1, the gradients g2 and
g1 that feed tensor-core products); every sum is carried in float64 here.
"""
from __future__ import annotations

import numpy as np

IN, HID = 8, 64
W1, B1 = 0, IN * HID
W2 = B1 + HID
B2 = W2 + HID * HID
W3 = B2 + HID
B3 = W3 + HID
NPARAM = B3 + 1
NNORM = 2 * IN + 2


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest, ties to even), as float64."""
    x = np.ascontiguousarray(x, np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(params: np.ndarray):
    p = np.asarray(params, np.float64)
    return (p[W1:B1].reshape(IN, HID), p[B1:W2], p[W2:B2].reshape(HID, HID), p[B2:W3],
            p[W3:B3], p[B3])


def forward_backward(params, norm, X, Y, bf=True):
    """Mean squared error of the normalised prediction and its gradient
    (flat, NPARAM) at `params`; norm = feature means[8], stds[8], target
    mean, target std."""
    r = bf16 if bf else (lambda a: np.asarray(a, np.float64))
    w1, b1, w2, b2, w3, b3 = unpack(params)
    norm = np.asarray(norm, np.float32)
    mean, inv_std = norm[:IN], (np.float32(1.0) / norm[IN:2 * IN])
    if bf:
        xn = ((np.asarray(X, np.float32) - mean) * inv_std).astype(np.float32)
    else:
        xn = (np.asarray(X, np.float64) - norm[:IN].astype(np.float64)) / norm[IN:2 * IN]
    x = r(xn)
    w1b, w2b = r(w1), r(w2)
    z1 = x @ w1b + b1
    h1 = r(np.maximum(z1, 0.0))
    z2 = h1 @ w2b + b2
    a2 = np.maximum(z2, 0.0)
    y = a2 @ w3 + b3
    t = (np.asarray(Y, np.float64) - norm[2 * IN]) / norm[2 * IN + 1]
    n = len(y)
    loss = float(np.mean((y - t) ** 2))
    dy = 2.0 * (y - t) / n
    g = np.zeros(NPARAM)
    g[W3:B3] = a2.T @ dy
    g[B3] = dy.sum()
    g2f = dy[:, None] * w3[None, :] * (z2 > 0)
    g[B2:W3] = g2f.sum(0)
    g2 = r(g2f)
    g[W2:B2] = (h1.T @ g2).ravel()
    dh1 = g2 @ w2b.T
    g1f = dh1 * (h1 > 0)
    g[B1:W2] = g1f.sum(0)
    g1 = r(g1f)
    g[W1:B1] = (x.T @ g1).ravel()
    return loss, g, y * norm[2 * IN + 1] + norm[2 * IN]


def init_params(seed: int = 0) -> np.ndarray:
    rng = np.random.Generator(np.random.PCG64(seed))
    p = np.zeros(NPARAM, np.float32)
    p[W1:B1] = rng.uniform(-1, 1, IN * HID) * np.sqrt(6 / IN)
    p[B1:W2] = rng.uniform(-0.1, 0.1, HID)
    p[W2:B2] = rng.uniform(-1, 1, HID * HID) * np.sqrt(6 / HID)
    p[B2:W3] = rng.uniform(-0.1, 0.1, HID)
    p[W3:B3] = rng.uniform(-1, 1, HID) * np.sqrt(6 / HID)
    p[B3] = 0.05
    return p
