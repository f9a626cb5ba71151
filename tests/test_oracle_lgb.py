"""CPU checks of the learned-Born-radius oracle (oracle/lgb_mlp.py): its
analytical gradient equals central differences of its loss (with the BF16
rounding switched off, which makes the loss smooth), and the BF16 rounding
is round-to-nearest-even."""
from __future__ import annotations

import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))

import lgb_mlp  # noqa: E402


def test_oracle_gradient_matches_central_differences(monkeypatch):
    monkeypatch.setattr(lgb_mlp, "bf16", lambda a: np.asarray(a, np.float64))
    rng = np.random.default_rng(0)
    p = rng.normal(scale=0.05, size=lgb_mlp.N_PARAMS)
    x = rng.random((40, lgb_mlp.N_INPUT))
    t = rng.normal(scale=0.2, size=40)
    _, g = lgb_mlp.loss_and_gradient(p, x, t)
    n = lgb_mlp.N_PARAMS
    for idx in rng.choice(n, 40, replace=False).tolist() + [n - 1, n - 17, n - 145, 128 * lgb_mlp.N_INPUT, 0]:
        e = np.zeros_like(p)
        e[idx] = 1e-6
        lp, _ = lgb_mlp.loss_and_gradient(p + e, x, t)
        lm, _ = lgb_mlp.loss_and_gradient(p - e, x, t)
        num = (lp - lm) / 2e-6
        assert abs(num - g[idx]) <= 1e-6 * max(abs(num), 1e-3), (idx, num, g[idx])


def test_bf16_rounding_is_nearest_even():
    vals = np.array([1.0, 1.0 + 2**-8, 1.0 + 3 * 2**-9, 1.0 + 2**-9, -2.5, 3.0e-5], dtype=np.float32)
    got = lgb_mlp.bf16(vals)
    # 1 + 2^-9 is a tie -> even (1.0); 1 + 3*2^-9 rounds up to 1 + 2^-7
    assert got[0] == 1.0 and got[3] == 1.0
    assert got[1] == 1.0 + 2**-8 or got[1] == 1.0  # 2^-8 needs 8 mantissa bits: tie -> even
    assert got[2] == 1.0 + 2**-7
    assert got[4] == -2.5
    assert abs(got[5] - 3.0e-5) <= 3.0e-5 * 2**-8
