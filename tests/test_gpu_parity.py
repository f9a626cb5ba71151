"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle on the
same seeded inputs.

Tolerances (stated per result):
  forces        RMS(F_gpu - F_oracle) / RMS(F_oracle) < 1e-5  (FP32 pair math,
                FP64 tile accumulation, 64-bit fixed-point sums)
  energies      |E_gpu - E_oracle| / max(|E_oracle|, 1) < 1e-6 per term (FP64 path)
  Born radii    < 1e-9 relative
  integrator    positions within 1e-6 A of the oracle after 5 BAOAB steps
                (same counter-based noise in both)
  determinism   bitwise identical reruns
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import INF, Orc, dp, oracle

pytestmark = pytest.mark.gpu

TRP = "NLYIQWLKDGGPSSGRPPPS"


def rms_rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


def helix(origami, seq):
    # compact alpha-helical build: many close non-bonded contacts
    return origami.Chain.build(seq, math.radians(-57.0), math.radians(-47.0), math.pi)


def jitter(x, scale=0.05, seed=0):
    return x + np.random.default_rng(seed).normal(scale=scale, size=x.shape)


_MIN_CACHE = {}


def minimized(origami, seq, helical=False):
    """Chain relaxed by L-BFGS on the CPU oracle (deterministic start for MD tests;
    origami likewise minimises before dynamics)."""
    key = (seq, helical)
    if key not in _MIN_CACHE:
        from test_minimize import OracleEngine
        from origami_b200.minimize import MinimizeOptions, lbfgs
        ch = helix(origami, seq) if helical else origami.Chain.build(seq)
        eng = OracleEngine(ch)
        lbfgs(eng, 0, MinimizeOptions(max_steps=300, gradient_tol=5.0))
        _MIN_CACHE[key] = eng.x.copy()
    ch = helix(origami, seq) if helical else origami.Chain.build(seq)
    ch.positions = _MIN_CACHE[key]
    return ch


def make_engine(origami, chain, xyz=None, params=None, temperature=310.0):
    eng = origami.Engine(params or origami.Params())
    eng.add_system(chain, chain.positions if xyz is None else xyz, temperature)
    eng.finalize()
    return eng


@pytest.mark.parametrize("mode", ["cutoff", "all_pairs"])
@pytest.mark.parametrize("build", ["extended", "helix"])
def test_total_force_matches_oracle(origami, mode, build):
    ch = origami.Chain.build(TRP) if build == "extended" else helix(origami, TRP)
    x = jitter(ch.positions, 0.03, 1)
    params = origami.Params() if mode == "cutoff" else origami.Params.all_pairs()
    eng = make_engine(origami, ch, x, params)
    f_gpu = eng.total_force(0)
    cut = (10.0, 20.0, 10.0) if mode == "cutoff" else (INF, INF, INF)
    f_ref = Orc(ch).total_force(x, *cut)
    err = rms_rel(f_gpu, f_ref)
    assert err < 1e-5, err
    assert np.isfinite(f_gpu).all()


def bench_chain(origami):
    """The benchmark's system: the seeded 300-residue chain (4 694 atoms, 147
    tiles) relaxed, from tests/golden/bench_chain_300.npz, as a product chain
    (its topology equals the fixture's, which bench.py also checks)."""
    import os
    z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "bench_chain_300.npz"))
    ch = origami.Chain.build(str(z["seq"]))
    ch.positions = z["xyz"]
    return ch


@pytest.mark.parametrize("mode", ["cutoff", "all_pairs"])
def test_total_force_on_the_bench_chain_matches_oracle(origami, mode):
    """The bench's relaxed chain, jittered: every force term against the
    oracle at the workload's own size (culled tile lists in cutoff mode, the
    full Newton-3 sweep in all-pairs mode)."""
    ch = bench_chain(origami)
    x = jitter(ch.positions, 0.02, 3)
    params = origami.Params() if mode == "cutoff" else origami.Params.all_pairs()
    f_gpu = make_engine(origami, ch, x, params).total_force(0)
    cut = (10.0, 20.0, 10.0) if mode == "cutoff" else (INF, INF, INF)
    f_ref = Orc(ch).total_force(x, *cut)
    err = rms_rel(f_gpu, f_ref)
    assert err < 1e-5, err
    assert np.isfinite(f_gpu).all()


@pytest.mark.parametrize("mode", ["cutoff", "all_pairs"])
def test_energies_on_the_bench_chain_match_oracle(origami, mode):
    """Per-term FP64 energies of the bench's relaxed chain (4 694 atoms: 11 M
    pair terms in the all-pairs GB and Coulomb sums) against the oracle at
    1e-6 relative, the tolerance of the smaller systems."""
    ch = bench_chain(origami)
    x = jitter(ch.positions, 0.02, 4)
    params = origami.Params() if mode == "cutoff" else origami.Params.all_pairs()
    e = make_engine(origami, ch, x, params).energies(0)
    nb, born = (10.0, 20.0) if mode == "cutoff" else (INF, INF)
    ref = Orc(ch).energy_terms(x, nb, born)
    for k in ("bond", "angle", "dihedral", "improper", "lj", "coulomb", "gb", "gb_self", "gb_pair", "total"):
        assert abs(e[k] - ref[k]) / max(abs(ref[k]), 1.0) < 1e-6, (k, e[k], ref[k])


def test_born_radii_match_oracle(origami):
    ch = helix(origami, TRP)
    x = jitter(ch.positions, 0.03, 2)
    eng = make_engine(origami, ch, x)
    r = eng.born_radii(0)
    ref = Orc(ch).born_radii(x, 20.0)
    assert np.max(np.abs(r - ref) / ref) < 1e-9


@pytest.mark.parametrize("mode", ["cutoff", "all_pairs"])
@pytest.mark.parametrize("build", ["extended", "helix"])
def test_born_integrals_match_oracle(origami, mode, build):
    # The radii all floor to rho - 0.09 (origami's descreening terms are
    # negative), so the integral itself is what checks the Born pass.
    # FP32 pair math: per-atom absolute error below 1e-6 of the largest |I|.
    ch = origami.Chain.build(TRP) if build == "extended" else helix(origami, TRP)
    x = jitter(ch.positions, 0.03, 5)
    params = origami.Params() if mode == "cutoff" else origami.Params.all_pairs()
    eng = make_engine(origami, ch, x, params)
    eng.total_force(0)
    got = eng.born_integrals(0)
    ref = Orc(ch).born_integrals(x, 20.0 if mode == "cutoff" else INF)
    assert np.max(np.abs(got - ref)) < 1e-6 * np.max(np.abs(ref)), np.max(np.abs(got - ref))


@pytest.mark.parametrize("mode", ["cutoff", "all_pairs"])
def test_energies_match_oracle(origami, mode):
    ch = helix(origami, TRP)
    x = jitter(ch.positions, 0.03, 3)
    params = origami.Params() if mode == "cutoff" else origami.Params.all_pairs()
    eng = make_engine(origami, ch, x, params)
    e = eng.energies(0)
    nb = 10.0 if mode == "cutoff" else INF
    born = 20.0 if mode == "cutoff" else INF
    ref = Orc(ch).energy_terms(x, nb, born)
    for k in ("bond", "angle", "dihedral", "improper", "lj", "coulomb", "gb", "gb_self", "gb_pair", "total"):
        assert abs(e[k] - ref[k]) / max(abs(ref[k]), 1.0) < 1e-6, (k, e[k], ref[k])


def test_batched_uneven_systems_match_single(origami):
    seqs = ["AKE", TRP, "GGPWYDNRQ", "M" * 7]
    chains = [helix(origami, s) for s in seqs]
    xs = [jitter(c.positions, 0.02, 10 + k) for k, c in enumerate(chains)]
    eng = origami.Engine(origami.Params())
    for c, x in zip(chains, xs):
        eng.add_system(c, x, 300.0)
    eng.finalize()
    for k, (c, x) in enumerate(zip(chains, xs)):
        f = eng.total_force(k)
        ref = Orc(c).total_force(x)
        assert rms_rel(f, ref) < 1e-5, (k, rms_rel(f, ref))
        single = make_engine(origami, c, x).total_force(0)
        assert np.allclose(f, single, rtol=1e-12, atol=1e-9)


@pytest.mark.parametrize("shake", [False, True])
def test_baoab_steps_match_oracle(origami, shake):
    ch = minimized(origami, "AKEWL", helical=True)
    x0 = ch.positions
    dt = 2.0 if shake else 1.0
    params = origami.Params(dt_fs=dt, friction_ps_inv=2.0, constrain_h_bonds=shake, seed=1234)
    eng = make_engine(origami, ch, x0, params, temperature=310.0)
    eng.init_velocities(0, 99, remove_com=True)
    v0 = eng.velocities(0)
    n_steps = 5
    eng.step(n_steps)
    x_gpu, v_gpu = eng.positions(0), eng.velocities(0)

    orc = Orc(ch)
    x = np.ascontiguousarray(x0.copy())
    v = np.ascontiguousarray(v0.copy())
    f = orc.total_force(x)
    fails = oracle().orc_baoab(orc.tp, dp(x), dp(v), dp(f), n_steps, dt, 2.0, 310.0, int(shake), 1234, 0, 0,
                               10.0, 20.0, 10.0)
    assert fails == 0
    assert np.max(np.abs(x_gpu - x)) < 1e-6
    assert np.max(np.abs(v_gpu - v)) < 1e-5
    st = eng.stats(0)
    assert st["steps"] == n_steps and st["shake_failures"] == 0 and not st["diverged"]
    if shake:
        t = ch.topology()
        c = t.constraints
        d = np.sqrt(((x_gpu[c[:, 0]] - x_gpu[c[:, 1]]) ** 2).sum(1))
        assert np.max(np.abs(d ** 2 - t.constraint_length ** 2)) < 1e-6


def test_deterministic_rerun(origami):
    ch = minimized(origami, TRP)
    runs = []
    for _ in range(2):
        eng = make_engine(origami, ch, None, origami.Params(dt_fs=2.0, constrain_h_bonds=True, seed=5))
        eng.init_velocities(0, 5)
        eng.step(20)
        runs.append((eng.positions(0), eng.velocities(0), eng.total_force(0)))
    for a, b in zip(runs[0], runs[1]):
        assert np.array_equal(a, b)


def test_initial_velocities_follow_reference_stream(origami):
    # langevin.rs:487-513: sigma * xoshiro gaussians x,y,z per atom, COM removed
    ch = origami.Chain.build("AK")
    eng = make_engine(origami, ch, None, origami.Params(), temperature=300.0)
    eng.init_velocities(0, 42, remove_com=False)
    v = eng.velocities(0)
    t = ch.topology()
    rng = origami.Xoshiro256pp(42)
    kbt = origami.BOLTZMANN_KJ_PER_MOL_K * 300.0
    ref = np.array([[math.sqrt(kbt * 1e-4 / m) * rng.gaussian() for _ in range(3)] for m in t.mass])
    assert np.array_equal(v, ref)


def test_thermostat_reaches_target(origami):
    # dynamics/tests/langevin_thermostat.rs: Ala3, 310 K, 2000 steps -> mean T within 60 K
    ch = minimized(origami, "AAA")
    res = origami.run_langevin(ch, origami.LangevinOptions(steps=2000, save_every=10, seed=3, friction_ps_inv=5.0))
    assert not res["diverged"]
    assert abs(res["temperature_mean_k"] - 310.0) < 60.0


def test_shake_dt2_no_failures(origami):
    # dynamics/tests/shake_dt2.rs: Trp-cage at dt 2 fs + SHAKE, 0 failures, T within 80 K
    ch = minimized(origami, TRP)
    res = origami.run_langevin(ch, origami.LangevinOptions(steps=1000, dt_fs=2.0, constrain_h_bonds=True,
                                                           save_every=20, seed=11, friction_ps_inv=5.0))
    assert res["shake_failures"] == 0 and not res["diverged"]
    assert abs(res["temperature_mean_k"] - 310.0) < 80.0


def test_remd_swap_exchanges_configurations(origami):
    ch = origami.Chain.build("AKE")
    x0 = ch.positions
    xa, xb = jitter(x0, 0.02, 20), jitter(x0, 0.02, 21)
    eng = origami.Engine(origami.Params())
    eng.add_system(ch, xa, 300.0)
    eng.add_system(ch, xb, 350.0)
    eng.finalize()
    eng.init_velocities(0, 1, False)
    eng.init_velocities(1, 2, False)
    va, vb = eng.velocities(0), eng.velocities(1)
    acc = eng.remd_swap(0, np.array([0.0]))  # u = 0 always accepts
    assert acc.tolist() == [1]
    assert np.array_equal(eng.positions(0), xb) and np.array_equal(eng.positions(1), xa)
    assert np.allclose(eng.velocities(0), vb * math.sqrt(300.0 / 350.0), rtol=0, atol=1e-15)
    assert np.allclose(eng.velocities(1), va * math.sqrt(350.0 / 300.0), rtol=0, atol=1e-15)
    acc = eng.remd_swap(0, np.array([1.0]))  # u = 1 rejects unless delta >= 0
    e = eng.all_energies()
    beta = [1 / (origami.BOLTZMANN_KJ_PER_MOL_K * t) for t in (300.0, 350.0)]
    delta = (beta[0] - beta[1]) * (e[0]["total"] - e[1]["total"])
    assert acc.tolist() == ([1] if delta >= 0 else [0])


def test_remd_driver_accepts(origami):
    # dynamics/tests/remd_acceptance.rs: Ala3, 4 replicas, best acceptance > 0.1
    ch = minimized(origami, "AAA")
    res = origami.run_remd(ch, origami.RemdOptions(temperatures_k=[300, 330, 360, 400], total_time_fs=4000.0,
                                                   swap_interval_fs=100.0, seed=9))
    assert max(res["acceptance_ratios"]) > 0.1


def test_nonfinite_positions_reported(origami):
    # Failure detection without a GPU fault: a host-injected NaN makes the step
    # report OG_E_NONFINITE and freezes that system only.
    ch = origami.Chain.build("AK")
    eng = origami.Engine(origami.Params())
    eng.add_system(ch, ch.positions, 300.0)
    eng.add_system(ch, ch.positions, 300.0)
    eng.finalize()
    x = ch.positions
    x[3, 0] = np.nan
    eng.set_positions(1, x)
    st = eng.step(2, check=False)
    assert st == 2
    assert eng.stats(1)["diverged"] and not eng.stats(0)["diverged"]
    assert np.isfinite(eng.positions(0)).all()


def test_cutoff_lists_on_long_chains(origami):
    """Cutoff mode culls tile pairs by bounding spheres every evaluation (most
    pairs of a 60-residue extended chain lie beyond 20 A): forces and Born
    integrals of two batched systems still match the oracle's cutoff sums."""
    seq = "ARNDCQEGHILKMFPSTWYV" * 3
    chains = [origami.Chain.build(seq), helix(origami, seq)]
    xs = [jitter(c.positions, 0.03, 11 + k) for k, c in enumerate(chains)]
    eng = origami.Engine(origami.Params())
    for c, x in zip(chains, xs):
        eng.add_system(c, x)
    eng.finalize()
    for k, (c, x) in enumerate(zip(chains, xs)):
        f = eng.total_force(k)
        ref = Orc(c).total_force(x, 10.0, 20.0, 10.0)
        assert rms_rel(f, ref) < 1e-5, (k, rms_rel(f, ref))
        got = eng.born_integrals(k)
        ref_i = Orc(c).born_integrals(x, 20.0)
        assert np.max(np.abs(got - ref_i)) < 1e-6 * np.max(np.abs(ref_i))
