"""L-BFGS host driver (origami_b200/minimize.py) against origami's minimiser
acceptance tests.  The CPU test drives it with the oracle standing in for the
engine; the GPU test drives the real engine through the C ABI."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import INF, Orc, dp, oracle, known
from origami_b200.minimize import MinimizeOptions, lbfgs

TRP = "NLYIQWLKDGGPSSGRPPPS"


class OracleEngine:
    """Engine-shaped wrapper over the CPU oracle for one chain."""

    def __init__(self, chain):
        self.orc = Orc(chain)
        self.x = np.ascontiguousarray(chain.positions)

    def positions(self, s):
        return self.x.copy()

    def set_positions(self, s, x):
        self.x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1, 3)

    def energies(self, s):
        return self.orc.energy_terms(self.x)

    def total_force(self, s):
        return self.orc.total_force(self.x)


def test_lbfgs_trp_cage_on_oracle(origami):
    # dynamics/tests/trp_cage_minimise.rs: extended Trp-cage -> < 1000 kJ/mol in
    # < 500 steps (gradient_tol 5), bond term < 200 kJ/mol afterwards.
    ch = origami.Chain.build(TRP)
    eng = OracleEngine(ch)
    res = lbfgs(eng, 0, MinimizeOptions(max_steps=500, gradient_tol=5.0, max_step_a=0.1))
    assert res.final_energy < known("trp_cage_minimised_total_below_kj"), res
    assert res.steps < known("trp_cage_minimise_steps_below"), res
    e = np.zeros(4)
    oracle().orc_bonded_energy(eng.orc.tp, dp(eng.x), dp(e))
    assert e[0] < known("trp_cage_minimised_bond_below_kj")
    assert res.initial_energy > 40000.0


def test_lbfgs_two_atoms_like_reference(origami):
    # lbfgs.rs lbfgs_ala3_chain_drops_below_sd_in_fewer_steps: energy decreases
    ch = origami.Chain.build("AAA")
    eng = OracleEngine(ch)
    res = lbfgs(eng, 0, MinimizeOptions(max_steps=200, gradient_tol=5.0))
    assert res.final_energy < res.initial_energy


@pytest.mark.gpu
def test_lbfgs_trp_cage_on_gpu(origami):
    from origami_b200.minimize import minimize_chain
    ch = origami.Chain.build(TRP)
    res = minimize_chain(ch, opts=MinimizeOptions(max_steps=500, gradient_tol=5.0))
    assert res.final_energy < 1000.0 and res.steps < 500, res
    ref = Orc(ch).energy_terms()
    assert abs(ref["total"] - res.final_energy) < 1e-6 * abs(ref["total"]) + 1e-6
    assert ref["bond"] < 200.0


class CountingQuartic:
    """Engine-shaped deterministic test function: E = sum k |x - c|^2 +
    b |x - c|^4 per atom plus a weak pair coupling; counts evaluations."""

    def __init__(self, n=40, seed=2):
        rng = np.random.default_rng(seed)
        self.c = rng.normal(size=(n, 3))
        self.x = self.c + rng.normal(scale=2.0, size=(n, 3))
        self.n_grad = self.n_energy = 0

    def positions(self, s):
        return self.x.copy()

    def set_positions(self, s, x):
        self.x = np.array(x, dtype=np.float64).reshape(-1, 3)

    def _terms(self):
        d = self.x - self.c
        r2 = (d * d).sum(axis=1)
        s = self.x.sum(axis=0)
        return d, r2, s

    def energies(self, s):
        self.n_energy += 1
        d, r2, sm = self._terms()
        return {"total": float((3.0 * r2 + 0.2 * r2 * r2).sum() + 0.01 * (sm * sm).sum())}

    def total_force(self, s):
        self.n_grad += 1
        d, r2, sm = self._terms()
        g = (6.0 + 0.8 * r2)[:, None] * d + 0.02 * sm[None, :]
        return -g


def _lbfgs_as_reference(engine, o):
    """lbfgs.rs:61-254 step by step: gradient at the top of every iteration,
    energy before every line search."""
    from collections import deque
    from origami_b200.minimize import _backtracking, _norm, _System, _two_loop
    S = _System(engine, 0)
    e_prev = S.energy()
    hs, hy, hr = deque(), deque(), deque()
    for step in range(o.max_steps):
        g = S.grad()
        max_force = _norm(g, o.gradient_norm)
        if max_force < o.gradient_tol:
            return step
        direction = -g if not hs else _two_loop(g, hs, hy, hr)
        md = float(np.max(np.abs(direction)))
        a0 = min(o.alpha0, o.max_step_a / md) if md > 0 else o.alpha0
        x = S.x()
        e_now = S.energy()
        res = _backtracking(S, x, direction, g, e_now, a0, o)
        if res is None:
            sd = -g
            md2 = float(np.max(np.abs(sd)))
            res2 = _backtracking(S, x, sd, g, e_now, min(o.alpha0, o.max_step_a / md2), o)
            if res2 is None:
                return step
            S.set_x(x + res2[0] * sd)
            hs.clear(); hy.clear(); hr.clear()
            e_prev = res2[1]
            continue
        alpha, e_new = res
        step_vec = alpha * direction
        S.set_x(x + step_vec)
        y = S.grad() - g
        sy = float(step_vec @ y)
        if sy > 1e-12:
            if len(hs) == o.history:
                hs.popleft(); hy.popleft(); hr.popleft()
            hs.append(step_vec); hy.append(y); hr.append(1.0 / sy)
        if abs(e_prev - e_new) < o.energy_tol and max_force < o.gradient_tol:
            return step + 1
        e_prev = e_new
    return o.max_steps - 1


def test_lbfgs_reuses_evaluations_without_changing_iterates():
    o = MinimizeOptions(max_steps=60, gradient_tol=1e-3, max_step_a=0.3)
    a, b = CountingQuartic(), CountingQuartic()
    res = lbfgs(a, 0, o)
    steps_ref = _lbfgs_as_reference(b, o)
    assert res.steps == steps_ref
    np.testing.assert_array_equal(a.x, b.x)
    assert a.n_grad < 0.6 * b.n_grad and a.n_energy < 0.75 * b.n_energy, (a.n_grad, b.n_grad, a.n_energy,
                                                                          b.n_energy)
