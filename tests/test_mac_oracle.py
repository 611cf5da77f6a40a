"""The learned-MAC network oracle's backward pass against finite differences
(float64, no BF16 rounding).  CPU only."""
from __future__ import annotations

import numpy as np

import mac_oracle as M


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.Generator(np.random.PCG64(3))
    p = M.init_params(1).astype(np.float64)
    norm = np.concatenate([rng.normal(0, 1, 8), rng.uniform(0.5, 2, 8), [1.0, 2.0]])
    X = rng.normal(0, 1.5, (64, 8))
    Y = rng.normal(1, 2, 64)
    _, g, _ = M.forward_backward(p, norm, X, Y, bf=False)
    idx = np.concatenate([rng.choice(M.B1, 10, replace=False),
                          M.B1 + rng.choice(64, 4, replace=False),
                          M.W2 + rng.choice(4096, 12, replace=False),
                          M.B2 + rng.choice(64, 4, replace=False),
                          M.W3 + rng.choice(64, 4, replace=False), [M.B3]])
    for i in idx:
        h = 1e-6 * max(1.0, abs(p[i]))
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        lp, _, _ = M.forward_backward(pp, norm, X, Y, bf=False)
        lm, _, _ = M.forward_backward(pm, norm, X, Y, bf=False)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-5 * max(1.0, abs(fd)), (i, fd, g[i])


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.3, 0.0], np.float32)
    r = M.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0078125 and r[4] == 0.0
    assert abs(r[3] + 3.3) < 0.02
