"""The learned-Born-radius network's GPU forward/backward (tensor-core GEMMs
+ head, SiLU and reduction kernels) against the NumPy oracle
(oracle/lgb_mlp.py) with the same BF16 rounding points, and a training run.

Tolerances: loss to 1e-4 relative; each parameter block's gradient to
3e-3 relative L2 (FP32 accumulation order and __expf in the SiLU can move an
intermediate across a BF16 rounding boundary)."""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))

import lgb_mlp  # noqa: E402

pytestmark = pytest.mark.gpu

def blocks():
    from origami_b200 import lgb
    o = [lgb.OFF_W1, lgb.OFF_B1, lgb.OFF_W2, lgb.OFF_B2, lgb.OFF_W3, lgb.OFF_B3, lgb.OFF_W4, lgb.OFF_B4, lgb.OFF_V,
         lgb.N_PARAMS]
    names = ("W1", "b1", "W2", "b2", "W3", "b3", "w4", "b4", "v")
    return [(names[k], o[k], o[k + 1]) for k in range(9)]


def data(n, seed):
    """Samples drawn with `seed` from one fixed smooth target function."""
    a = np.random.default_rng(1234).normal(size=80) / 8.0
    rng = np.random.default_rng(seed)
    x = np.log1p(rng.gamma(2.0, 1.5, size=(n, 80))).astype(np.float32)
    t = (0.4 * np.tanh(x @ a - 2.0) - 0.1).astype(np.float32)
    return x, t


@pytest.mark.parametrize("n", [300, 1024])
def test_gradient_matches_oracle(origami, n):
    from origami_b200 import lgb
    x, t = data(n, n)
    p = lgb.init_params(3)
    p[lgb.OFF_B1:lgb.OFF_W2] = np.random.default_rng(1).normal(scale=0.1, size=128)
    p[lgb.OFF_V:] = np.random.default_rng(2).normal(scale=0.1, size=lgb.N_SELF)
    # non-zero output weights, so every layer's gradient is exercised
    p[lgb.OFF_W4:lgb.OFF_B4] = np.random.default_rng(3).normal(scale=0.1, size=128)
    loss, g = lgb.loss_and_gradient(x, t, p)
    loss_ref, g_ref = lgb_mlp.loss_and_gradient(p, x, t)
    assert abs(loss - loss_ref) <= 1e-4 * loss_ref
    for name, a, b in blocks():
        num = np.linalg.norm(g[a:b] - g_ref[a:b])
        den = np.linalg.norm(g_ref[a:b])
        assert num <= 3e-3 * den + 1e-12, (name, num / den)


def test_training_reduces_loss(origami):
    from origami_b200 import lgb
    x, t = data(20000, 7)
    p0 = lgb.init_params(11)
    p, hist = lgb.train(x, t, p0, steps=600, batch=1024, lr=2e-3, seed=5)
    assert np.isfinite(hist).all()
    first, last = float(hist[:20].mean()), float(hist[-50:].mean())
    assert last < 0.1 * first, (first, last)
    # the trained parameters evaluate to the reported loss on held-out rows
    xv, tv = data(4000, 8)
    lv, _ = lgb.loss_and_gradient(xv, tv, p)
    assert lv < 0.2 * first
    assert not np.array_equal(p, p0)
