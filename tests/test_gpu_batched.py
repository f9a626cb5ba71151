"""Batched uneven systems on one GPU: the pair passes' launch variants
(og_engine_set_pair_launch), the autotuner and its cache
(og_engine_autotune), the 256-chain batch of uneven lengths (residues
U[10, 80], seeded), and parallel tempering with device-side swaps
(og_remd_run) -- origami's replica loop (dynamics/src/remd.rs:286,
replicas.par_iter_mut()) and swap rule (remd.rs:425-474) on the device.

Tolerances: forces RMS relative < 1e-5 against the FP64 oracle for every
variant; a persistent launch and a one-CTA-per-item launch of the same shape
and chunk give bit-identical forces (each item's sums are the same, and
fixed-point accumulation makes the order irrelevant).
"""
from __future__ import annotations

import math
import os
import sys

import numpy as np
import pytest

from conftest import INF, Orc

pytestmark = pytest.mark.gpu


def rms_rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


def _bench():
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    return bench


def _jitter(x, s, seed):
    return x + np.random.default_rng(seed).normal(scale=s, size=x.shape)


def _uneven_batch(origami, params):
    seqs = ["GYDPETGTWG", "NLYIQWLKDGGPSSGRPPPS" * 2, "AKE", "ARNDCQEGHILKMFPSTWYV" * 3]
    chains = [origami.Chain.build(s, math.radians(-57.0), math.radians(-47.0), math.pi) if k % 2 else
              origami.Chain.build(s) for k, s in enumerate(seqs)]
    xs = [_jitter(c.positions, 0.03, 40 + k) for k, c in enumerate(chains)]
    eng = origami.Engine(params)
    for c, x in zip(chains, xs):
        eng.add_system(c, x, 300.0)
    eng.finalize()
    return eng, chains, xs


@pytest.mark.parametrize("mode", ["all_pairs", "cutoff"])
def test_pair_launch_variants_match_oracle(origami, mode):
    params = origami.Params.all_pairs() if mode == "all_pairs" else origami.Params()
    cut = (INF, INF, INF) if mode == "all_pairs" else (10.0, 20.0, 10.0)
    eng, chains, xs = _uneven_batch(origami, params)
    refs = [Orc(c).total_force(x, *cut) for c, x in zip(chains, xs)]
    for shape in (0, 1, 2, 3, 4, 5, 6):
        for chunk in (8, 32):
            got = {}
            for persistent in (False, True):
                eng.set_pair_launch("born", min(shape, 2), persistent, chunk)
                eng.set_pair_launch("force", shape, persistent, chunk)
                fs = [eng.total_force(k) for k in range(len(chains))]
                for k, (f, ref) in enumerate(zip(fs, refs)):
                    assert rms_rel(f, ref) < 1e-5, (shape, persistent, chunk, k, rms_rel(f, ref))
                got[persistent] = fs
            for a, b in zip(got[False], got[True]):
                assert np.array_equal(a, b), (shape, chunk)


def test_autotune_picks_a_variant_and_caches_it(origami, tmp_path):
    cache = str(tmp_path / "tune.json")
    eng, chains, xs = _uneven_batch(origami, origami.Params.all_pairs())
    r = eng.autotune(cache)
    assert r["from_cache"] == 0
    assert 0 <= r["born_shape"] <= 2 and 0 <= r["force_shape"] <= 6
    assert r["born_chunk"] in (8, 16, 32) and r["force_chunk"] in (8, 16, 32)
    # the chosen variant is the fastest timed, so no slower than the default
    assert r["born_ms"] <= r["born_ms_default"] and r["force_ms"] <= r["force_ms_default"]
    for k, (c, x) in enumerate(zip(chains, xs)):
        assert rms_rel(eng.total_force(k), Orc(c).total_force(x, INF, INF, INF)) < 1e-5
    eng.close()
    eng2, _, _ = _uneven_batch(origami, origami.Params.all_pairs())
    r2 = eng2.autotune(cache)
    assert r2["from_cache"] == 1
    for key in ("born_shape", "born_persistent", "born_chunk", "force_shape", "force_persistent", "force_chunk"):
        assert r2[key] == r[key]
    text = open(cache).read()
    assert "all_pairs|tiles<=" in text


def test_c3b_batch_of_256_uneven_chains(origami):
    """The 256-chain workload: residue counts U[10, 80] (seeded), each chain
    a separate system at 310 K, GB only, all pairs.  Every system's forces
    against the oracle after autotuning, then MD at dt 2 fs + SHAKE."""
    bench = _bench()
    seqs = bench.c3b_sequences(0)
    assert len(seqs) == 256 and min(map(len, seqs)) >= 10 and max(map(len, seqs)) <= 80
    chains = [origami.Chain.build(s) for s in seqs]
    xs = [_jitter(c.positions, 0.02, 1000 + k) for k, c in enumerate(chains)]
    eng = origami.Engine(origami.Params.all_pairs(dt_fs=2.0, friction_ps_inv=2.0, constrain_h_bonds=True, seed=5))
    for c, x in zip(chains, xs):
        eng.add_system(c, x, 310.0)
    eng.finalize()
    eng.autotune(None)
    worst = 0.0
    for k, (c, x) in enumerate(zip(chains, xs)):
        err = rms_rel(eng.total_force(k), Orc(c).total_force(x, INF, INF, INF))
        worst = max(worst, err)
    assert worst < 1e-5, worst
    # relax every chain at once (the extended builds carry bond strain),
    # then MD
    from origami_b200.minimize import MinimizeOptions, minimize_all
    for k in range(len(chains)):
        eng.set_positions(k, chains[k].positions)
    res = minimize_all(eng, MinimizeOptions(max_steps=400, gradient_tol=5.0))
    assert res.final_energy < res.initial_energy
    for k in range(len(chains)):
        eng.init_velocities(k, 77 + k, remove_com=False)
    eng.step(100)
    for k in range(len(chains)):
        st = eng.stats(k)
        assert not st["diverged"] and st["shake_failures"] == 0 and st["steps"] == 100


def test_device_remd_rounds(origami):
    """og_remd_run: the ladder is kept (each temperature held by exactly one
    system, the system's own temperature equal to its slot's), attempts
    follow the even/odd schedule, neighbouring temperatures exchange, and a
    rerun with the same seed makes the same decisions."""
    from test_gpu_parity import minimized
    ch = minimized(origami, "AAAK")
    temps = [280.0 * (1.5 ** (k / 5)) for k in range(6)]  # geometric 280 .. 420 K
    runs = []
    for _ in range(2):
        eng = origami.Engine(origami.Params(dt_fs=2.0, friction_ps_inv=2.0, constrain_h_bonds=True, seed=3))
        for t in temps:
            eng.add_system(ch, ch.positions, t)
        eng.finalize()
        for k in range(len(temps)):
            eng.init_velocities(k, 11 + k, remove_com=False)
        r = eng.remd_run(20, 50, 99)
        slots = r["sys_of_slot"]
        assert sorted(slots.tolist()) == list(range(len(temps)))
        for k, sy in enumerate(slots):
            assert abs(eng.kinetic(int(sy))[1] - temps[k]) < 0.6 * temps[k]  # thermalised near its slot
        assert r["attempts"].tolist() == [10, 10, 10, 10, 10]  # pairs 0,2,4 on even rounds; 1,3 on odd
        assert r["accepts"].sum() > 0
        runs.append((slots.copy(), r["accepts"].copy(), eng.positions(0)))
        eng.close()
    assert np.array_equal(runs[0][0], runs[1][0]) and np.array_equal(runs[0][1], runs[1][1])
    assert np.array_equal(runs[0][2], runs[1][2])


def test_device_remd_equal_temperatures_always_exchange(origami):
    """Two systems at equal temperature: delta = 0, so the exchange is
    accepted whatever the energies, and the slots swap after one round."""
    from test_gpu_parity import minimized
    ch = minimized(origami, "AKE")
    eng = origami.Engine(origami.Params(seed=1))
    eng.add_system(ch, ch.positions, 300.0)
    eng.add_system(ch, ch.positions, 300.0)
    eng.finalize()
    eng.init_velocities(0, 1, False)
    eng.init_velocities(1, 2, False)
    r = eng.remd_run(1, 1, 7)
    assert r["attempts"].tolist() == [1] and r["accepts"].tolist() == [1]
    assert r["sys_of_slot"].tolist() == [1, 0]
