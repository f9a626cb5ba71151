"""Learned Born radii in the engine (born_mode = 1): descriptor and
Coulomb-field parity with the NumPy oracle, the radii the network produces,
the plain-GB judge and its fallback, and what a trained network gains over
the Coulomb-field estimate alone.

Tolerances: descriptors 2e-5 absolute on log(1 + D) (FP32 relative
coordinates and __expf); Coulomb-field radii 1e-5 relative; learned radii
R_cfa exp(b4) 1e-6 relative."""
from __future__ import annotations

import math
import os
import sys

import numpy as np
import pytest

from conftest import Orc

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))

import lgb_descriptors  # noqa: E402

pytestmark = pytest.mark.gpu

TRP = "NLYIQWLKDGGPSSGRPPPS"


def chains(origami):
    rng = np.random.default_rng(4)
    ext = origami.Chain.build(TRP)
    hel = origami.Chain.build(TRP, math.radians(-57.0), math.radians(-47.0), math.pi)
    big = origami.Chain.build("ARNDCQEGHILKMFPSTWYV" * 3)
    return [(ext, ext.positions), (hel, hel.positions + rng.normal(scale=0.03, size=hel.positions.shape)),
            (big, big.positions)]


def oracle_inputs(chain, x):
    t = chain.topology()
    rho = np.asarray(t.gb_rho)
    rt = rho - 0.09
    return lgb_descriptors.descriptors(x, np.asarray(t.element), rho, rt, np.asarray(t.gb_scale) * rt)


def test_descriptors_and_targets_match_oracle(origami):
    from origami_b200 import lgb
    rows = chains(origami)
    eng = origami.Engine(origami.Params())
    for ch, x in rows:
        eng.add_system(ch, x)
    eng.finalize()
    for k, (ch, x) in enumerate(rows):
        xin, target = lgb.samples(eng, k)
        x_ref, rcfa_ref = oracle_inputs(ch, x)
        assert np.abs(xin - x_ref).max() < 2e-5, np.abs(xin - x_ref).max()
        r_plain = Orc(ch).born_radii(x)
        t_ref = np.log(r_plain / rcfa_ref)
        assert np.abs(target - t_ref).max() < 1e-5, np.abs(target - t_ref).max()


def constant_params(origami, b4):
    from origami_b200 import lgb
    p = lgb.init_params(1)
    p[lgb.OFF_W4:lgb.OFF_B4] = 0.0
    p[lgb.OFF_B4] = b4
    p[lgb.OFF_V:] = 0.0
    return p


def learned_engine(origami, rows, params, judge=0, tol=1e-3):
    from origami_b200 import lgb
    p = origami.Params()
    p.born_mode = 1
    eng = origami.Engine(p)
    for ch, x in rows:
        eng.add_system(ch, x)
    eng.finalize()
    lgb.set_params(eng, params)
    lgb.set_judge(eng, judge, tol)
    return eng


def test_learned_radii_are_cfa_times_exp_output(origami):
    rows = chains(origami)
    eng = learned_engine(origami, rows, constant_params(origami, 0.25))
    for k, (ch, x) in enumerate(rows):
        _, rcfa = oracle_inputs(ch, x)
        got = eng.born_radii(k)
        np.testing.assert_allclose(got, rcfa * math.exp(np.float32(0.25)), rtol=1e-5)
        assert np.isfinite(eng.total_force(k)).all()


def random_params(origami, seed):
    from origami_b200 import lgb
    rng = np.random.default_rng(seed)
    p = lgb.init_params(seed)
    p[lgb.OFF_B1:lgb.OFF_W2] = rng.normal(scale=0.1, size=128)
    p[lgb.OFF_W4:lgb.OFF_B4] = rng.normal(scale=0.05, size=128)
    p[lgb.OFF_B4] = -0.1
    p[lgb.OFF_V:] = rng.normal(scale=0.05, size=lgb.N_SELF)
    return p


def test_fused_network_matches_layers_and_oracle(origami, monkeypatch):
    """The fused tensor-core kernel against the three GEMM layers + head
    (same rounding points: 1e-5) and against the NumPy network on the
    engine's own inputs (BF16 rounding of operands emulated: 2e-3)."""
    import lgb_mlp
    from origami_b200 import lgb
    rows = chains(origami)
    params = random_params(origami, 9)
    fused = learned_engine(origami, rows, params)
    monkeypatch.setenv("OG_LGB_UNFUSED", "1")
    layered = learned_engine(origami, rows, params)
    for k, (ch, x) in enumerate(rows):
        r_f, r_l = fused.born_radii(k), layered.born_radii(k)
        np.testing.assert_allclose(r_f, r_l, rtol=1e-5)
        xin, target = lgb.samples(fused, k)
        rcfa = Orc(ch).born_radii(x) / np.exp(target.astype(np.float64))
        y = np.clip(lgb_mlp.forward(params, xin)["y"], -5.0, 5.0)
        np.testing.assert_allclose(r_f, rcfa * np.exp(y), rtol=2e-3)


def test_engine_requires_parameters(origami):
    p = origami.Params()
    p.born_mode = 1
    eng = origami.Engine(p)
    ch, x = chains(origami)[0]
    eng.add_system(ch, x)
    eng.finalize()
    with pytest.raises(origami.OrigamiError) as e:
        eng.step(1)
    assert "og_lgb_set_params" in str(e.value)


def test_judge_falls_back_to_plain_gb(origami):
    from origami_b200 import lgb
    rows = chains(origami)[:2]
    plain = origami.Engine(origami.Params())
    for ch, x in rows:
        plain.add_system(ch, x)
    plain.finalize()
    # radii three times the Coulomb-field estimate: far from plain GB
    eng = learned_engine(origami, rows, constant_params(origami, math.log(3.0)), judge=0)
    err = lgb.judge(eng)
    st = lgb.status(eng)
    assert err > 1e-3 and not st["active"] and st["judged"] == 1
    for k in range(len(rows)):
        np.testing.assert_array_equal(eng.total_force(k), plain.total_force(k))
        np.testing.assert_array_equal(eng.born_radii(k), plain.born_radii(k))


def test_judge_runs_every_interval_during_steps(origami):
    from origami_b200 import lgb
    from test_gpu_parity import minimized
    ch = minimized(origami, TRP)
    eng = learned_engine(origami, [(ch, ch.positions)], constant_params(origami, 0.0), judge=5, tol=10.0)
    eng.init_velocities(0, 3, True)
    eng.step(12)
    st = lgb.status(eng)
    assert st["judged"] == 2 and st["active"] and st["last_error"] > 0.0


def test_trained_network_beats_coulomb_field_estimate(origami):
    """Samples from a short plain-GB trajectory of several chains; after
    training, the learned radii's GB forces are closer to plain GB than the
    Coulomb-field radii alone (the network with zero output)."""
    from origami_b200 import lgb
    from test_gpu_parity import minimized
    seqs = [TRP, "ARNDCQEGHILKMFPSTWYV", "GSAVKLEEIWDNRTQ"]
    chs = [minimized(origami, s) for s in seqs]
    p = origami.Params(dt_fs=2.0, constrain_h_bonds=True, seed=2)
    md = origami.Engine(p)
    for c in chs:
        md.add_system(c, c.positions)
    md.finalize()
    for k in range(len(chs)):
        md.init_velocities(k, 10 + k, True)
    xs, ts = [], []
    for _ in range(12):
        md.step(25)
        for k in range(len(chs)):
            x, t = lgb.samples(md, k)
            xs.append(x)
            ts.append(t)
    x, t = np.concatenate(xs), np.concatenate(ts)
    params, hist = lgb.train(x, t, lgb.init_params(7), steps=800, batch=2048, lr=2e-3, seed=1)
    assert hist[-50:].mean() < 0.05 * hist[:10].mean()

    rows = [(c, md.positions(k)) for k, c in enumerate(chs)]
    plain = origami.Engine(origami.Params())
    for c, xx in rows:
        plain.add_system(c, xx)
    plain.finalize()
    trained = learned_engine(origami, rows, params)
    baseline = learned_engine(origami, rows, constant_params(origami, 0.0))
    for k in range(len(rows)):
        f_ref = plain.total_force(k)
        err = lambda f: float(np.sqrt(((f - f_ref) ** 2).sum() / (f_ref ** 2).sum()))  # noqa: E731
        e_trained, e_base = err(trained.total_force(k)), err(baseline.total_force(k))
        assert e_trained < 0.5 * e_base, (k, e_trained, e_base)
