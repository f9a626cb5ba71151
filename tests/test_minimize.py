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
