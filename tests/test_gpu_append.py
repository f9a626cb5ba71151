"""Engines grown in place (og_engine_append_atoms) against engines built from
scratch and against the FP64 oracle.  A chain grows residue by residue as
the ribosome emits it (cotranslate.rs:204-231); after each append the grown
engine must give the forces of a fresh engine on the same state bit for bit
(fixed-point accumulation), the same energies, the same dynamics, and keep
the old atoms' velocities and the step count it had.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import INF, Orc, dp, oracle

pytestmark = pytest.mark.gpu

TERMS = ("bond", "angle", "dihedral", "improper", "lj", "coulomb", "gb", "sasa", "total")


def _fresh(origami, params, ch, x, v, steps):
    eng = origami.Engine(params)
    eng.add_system(ch, x)
    eng.finalize()
    eng.set_state({"velocities": np.ascontiguousarray(v), "steps": np.array([steps], dtype=np.int64)})
    return eng


@pytest.mark.parametrize("mode", ["all_pairs_sasa", "cutoff"])
def test_grown_engine_equals_a_fresh_one_residue_by_residue(origami, mode):
    if mode == "all_pairs_sasa":
        params = origami.Params.all_pairs(include_sasa=True, sasa_gamma_scale=0.25, constrain_h_bonds=True,
                                          dt_fs=2.0, seed=5)
    else:
        params = origami.Params(constrain_h_bonds=True, dt_fs=2.0, seed=5)
    rng = np.random.default_rng(3)
    ch = origami.Chain.build("MKT")
    eng = origami.Engine(params)
    eng.add_system(ch, ch.positions)
    eng.finalize()
    eng.init_velocities(0, 11)
    eng.step(3)
    steps = 3
    for aa in "WALDEKRYGHPSNFQC":  # 16 residues: the system crosses several 32-atom tiles
        ch.positions = eng.positions(0)
        v_before = eng.velocities(0)
        n_old = ch.n_atoms
        ch.append(aa)
        x = ch.positions
        v_new = rng.normal(scale=0.005, size=(ch.n_atoms - n_old, 3))
        eng.append_atoms(0, ch, x[n_old:], v_new)
        assert eng.n_atoms(0) == ch.n_atoms
        np.testing.assert_array_equal(eng.positions(0), x)
        v = eng.velocities(0)
        np.testing.assert_array_equal(v[:n_old], v_before)
        np.testing.assert_array_equal(v[n_old:], v_new)
        assert eng.stats(0)["steps"] == steps
        fresh = _fresh(origami, params, ch, x, v, steps)
        try:
            np.testing.assert_array_equal(eng.total_force(0), fresh.total_force(0))
            eg, ef = eng.energies(0), fresh.energies(0)
            for k in TERMS:
                assert abs(eg[k] - ef[k]) <= 1e-12 * max(abs(ef[k]), 1.0), (aa, k, eg[k], ef[k])
            eng.step(4)
            fresh.step(4)
            np.testing.assert_array_equal(eng.positions(0), fresh.positions(0))
            np.testing.assert_array_equal(eng.velocities(0), fresh.velocities(0))
            steps += 4
        finally:
            fresh.close()
    eng.close()


def test_grown_engine_matches_oracle_with_surface_term(origami):
    """A 60-residue chain grown by three residues: all-pairs forces with the
    surface term against the FP64 oracle (RMS relative < 1e-5)."""
    import bench
    seq = bench.seeded_sequence(63, 1)
    ch = origami.Chain.build(seq[:60])
    x0 = ch.positions + np.random.default_rng(8).normal(scale=0.02, size=(ch.n_atoms, 3))
    ch.positions = x0
    params = origami.Params.all_pairs(include_sasa=True, sasa_gamma_scale=0.25)
    eng = origami.Engine(params)
    eng.add_system(ch, x0)
    eng.finalize()
    for aa in seq[60:]:
        n_old = ch.n_atoms
        ch.append(aa)
        eng.append_atoms(0, ch, ch.positions[n_old:])
    x = np.ascontiguousarray(ch.positions)
    f = eng.total_force(0)
    eng.close()
    ref = Orc(ch).total_force(x, INF, INF, INF)
    o = oracle()
    el = ch.topology().element
    rad = np.array([o.orc_sasa_radius(int(e)) for e in el])
    gam = np.array([o.orc_sasa_gamma(int(e), 0.25) for e in el])
    fs = np.zeros_like(x)
    o.orc_sasa_forces_tangent_one_root(x.shape[0], dp(x), dp(rad), dp(gam), dp(fs))
    err = float(np.sqrt(((f - ref - fs) ** 2).sum() / ((ref + fs) ** 2).sum()))
    assert err < 1e-5, err


def test_learned_radii_engine_grows(origami):
    """With learned Born radii the network's per-atom buffers grow too: the
    grown engine's radii and forces equal a fresh engine's."""
    from origami_b200 import lgb
    from test_gpu_lgb import random_params
    p = random_params(origami, 4)
    params = origami.Params(born_mode=1)
    ch = origami.Chain.build("GAVLK")
    eng = origami.Engine(params)
    eng.add_system(ch, ch.positions)
    eng.finalize()
    lgb.set_params(eng, p)
    for aa in "DEWYF":
        n_old = ch.n_atoms
        ch.append(aa)
        eng.append_atoms(0, ch, ch.positions[n_old:])
    fresh = origami.Engine(params)
    fresh.add_system(ch, ch.positions)
    fresh.finalize()
    lgb.set_params(fresh, p)
    np.testing.assert_array_equal(eng.total_force(0), fresh.total_force(0))
    np.testing.assert_array_equal(eng.born_radii(0), fresh.born_radii(0))
    eng.close()
    fresh.close()


def test_append_refuses_what_does_not_extend(origami):
    ch = origami.Chain.build("GAV")
    eng = origami.Engine(origami.Params())
    eng.add_system(ch, ch.positions)
    eng.finalize()
    other = origami.Chain.build("GAVL")
    t = other.topology()
    t.charge[0] += 0.5
    with pytest.raises(origami.OrigamiError, match="parameters"):
        eng.append_atoms(0, t, other.positions[ch.n_atoms:])
    # the engine is unchanged and still usable
    assert eng.n_atoms(0) == ch.n_atoms
    assert np.isfinite(eng.total_force(0)).all()
    eng.close()


def test_cotranslation_grown_in_place_equals_rebuilt(origami):
    """The whole driver (append, L-BFGS, velocity seeding, slices with SHAKE
    and the tunnel) with grown engines and with engines rebuilt per slice:
    the same chain at the end."""
    from origami_b200.cotranslate import CotranslateTimings, CylindricalTunnel, UniformRibosome, run_cotranslate
    tun = CylindricalTunnel(axis_origin=(-5.0, 0.0, 0.0), axis_direction=(1.0, 0.0, 0.0), radius_a=10.0,
                            length_a=80.0, k_confine=10.0)
    opts = origami.LangevinOptions(dt_fs=2.0, temperature_k=310.0, friction_ps_inv=2.0, save_every=0, seed=7,
                                   include_sasa=True, constrain_h_bonds=True)
    params = origami.Params.all_pairs(sasa_gamma_scale=0.25)
    out = []
    for grow in (True, False):
        t = CotranslateTimings()
        ch = run_cotranslate(UniformRibosome("MGSKLTEW", 60.0), opts, 30, tun, params=params, timings=t,
                             grow_in_place=grow)
        assert t.slices == 8 and t.steps == 7 * 30 + 30
        out.append(ch.positions)
    assert out[0].shape == out[1].shape
    assert np.max(np.abs(out[0] - out[1])) < 1e-6


def test_last_of_several_systems_grows(origami):
    """Three systems in one engine, the last one grown: every system's
    forces equal those of engines built from scratch, the first two
    untouched; a system other than the last cannot grow."""
    params = origami.Params.all_pairs(include_sasa=True, sasa_gamma_scale=0.25)
    chains = [origami.Chain.build(s) for s in ("GAVLK", "MKTWE", "DEF")]
    eng = origami.Engine(params)
    for ch in chains:
        eng.add_system(ch, ch.positions)
    eng.finalize()
    before = [eng.total_force(k) for k in range(2)]
    last = chains[2]
    for aa in "RYHQNSTPC":  # several tiles' worth of atoms
        n_old = last.n_atoms
        last.append(aa)
        eng.append_atoms(2, last, last.positions[n_old:])
    with pytest.raises(origami.OrigamiError):
        grown0 = origami.Chain.build("GAVLK")
        grown0.append("A")
        eng.append_atoms(0, grown0, grown0.positions[chains[0].n_atoms:])
    for k, ch in enumerate(chains):
        fresh = origami.Engine(params)
        fresh.add_system(ch, ch.positions)
        fresh.finalize()
        np.testing.assert_array_equal(eng.total_force(k), fresh.total_force(0), err_msg=str(k))
        fresh.close()
    for k in range(2):
        np.testing.assert_array_equal(eng.total_force(k), before[k])
    eng.close()
