"""CPU: the surrogate network's FP64 oracle against finite differences."""
from __future__ import annotations

import numpy as np

from oracle import mlp_oracle as mo


def test_layout_total():
    L = mo.layout(41, 24)
    assert L["total"] == 128 * 41 + 128 + 2 * (128 * 128 + 128) + 24 * 128 + 24


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    n_in, n_out, n = 5, 3, 7
    p = mo.init_params(n_in, n_out, 1).astype(np.float64)
    p += rng.normal(0, 0.05, p.size)  # nonzero biases
    x = rng.normal(size=(n, n_in))
    t = rng.normal(size=(n, n_out))
    loss, g = mo.loss_grad(p, x, t, n_in, n_out, bf16_round=False)
    idx = rng.choice(p.size, 60, replace=False)
    h = 1e-6
    for i in idx:
        e = np.zeros_like(p)
        e[i] = h
        lp, _ = mo.loss_grad(p + e, x, t, n_in, n_out, bf16_round=False)
        lm, _ = mo.loss_grad(p - e, x, t, n_in, n_out, bf16_round=False)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])), i


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 2 ** -7 + 2 ** -8, -3.14159], dtype=np.float32)
    r = mo.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0                     # tie -> even
    assert r[2] == 1.0 + 2 ** -6           # tie -> even (odd mantissa rounds up)
    assert abs(r[3] + 3.140625) < 1e-12
