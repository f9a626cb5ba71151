"""Whole-engine state, checkpoints and trajectory capture on the GPU:
restoring a state (in memory or from a checkpoint file) continues a run bit
for bit; new positions without forces trigger a fresh force evaluation;
captured trajectory frames hold the positions of the steps they were taken
at (to the PDB's 3 decimals)."""
from __future__ import annotations

import numpy as np
import pytest

from test_gpu_parity import minimized

pytestmark = pytest.mark.gpu

SEQS = ["NLYIQWLKDGGPSSGRPPPS", "ARNDCQEGHILKMFPSTWYV"]


def make_engine(origami, sasa=False):
    chains = [minimized(origami, s) for s in SEQS]
    p = origami.Params(dt_fs=2.0, constrain_h_bonds=True, seed=5, include_sasa=sasa, sasa_gamma_scale=0.25)
    eng = origami.Engine(p)
    for k, c in enumerate(chains):
        eng.add_system(c, c.positions, 300.0 + 10.0 * k)
    eng.finalize()
    for k in range(len(chains)):
        eng.init_velocities(k, 40 + k, True)
    return eng, chains


def all_positions(eng):
    return [eng.positions(k) for k in range(eng.n_systems)]


@pytest.mark.parametrize("sasa", [False, True])
def test_state_round_trip_continues_bit_for_bit(origami, sasa):
    eng, _ = make_engine(origami, sasa)
    eng.step(20)
    st = eng.get_state()
    n, s = eng.counts()
    assert st["positions"].shape == (n, 3) and s == len(SEQS)
    assert list(st["steps"]) == [20, 20]
    eng.step(30)
    ref = all_positions(eng)
    ref_v = eng.get_state(parts=("velocities",))["velocities"].copy()
    eng.set_state(st)
    eng.step(30)
    got = all_positions(eng)
    for a, b in zip(ref, got):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(eng.get_state(parts=("velocities",))["velocities"], ref_v)


def test_checkpoint_file_restores_a_fresh_engine(origami, tmp_path):
    eng, _ = make_engine(origami)
    eng.step(15)
    eng.set_temperature(1, 350.0)
    path = str(tmp_path / "run.ckpt")
    eng.save_checkpoint(path)
    eng.step(25)
    ref = all_positions(eng)
    fresh, _ = make_engine(origami)
    fresh.load_checkpoint(path)
    assert fresh.temperature(1) == 350.0
    fresh.step(25)
    for a, b in zip(ref, all_positions(fresh)):
        np.testing.assert_array_equal(a, b)
    st = fresh.get_state(parts=("steps",))
    assert list(st["steps"]) == [40, 40]


def test_checkpoint_rejects_other_systems(origami, tmp_path):
    eng, _ = make_engine(origami)
    path = str(tmp_path / "run.ckpt")
    eng.save_checkpoint(path)
    other = origami.Engine(origami.Params())
    c = minimized(origami, SEQS[0])
    other.add_system(c, c.positions)
    other.finalize()
    with pytest.raises(origami.OrigamiError):
        other.load_checkpoint(path)
    bad = tmp_path / "bad.ckpt"
    bad.write_bytes(b"not a checkpoint at all")
    with pytest.raises(origami.OrigamiError):
        eng.load_checkpoint(str(bad))


def test_new_positions_without_forces_are_evaluated(origami):
    """Positions restored alone invalidate the cached forces: the next step
    starts from forces at the new positions, exactly as after set_positions."""
    a, _ = make_engine(origami)
    b, _ = make_engine(origami)
    a.step(10)
    b.step(10)
    st = a.get_state(parts=("positions", "velocities"))
    x = st["positions"].copy()
    x[:5] += 0.01
    a.set_state({"positions": x})
    off = 0
    for k in range(b.n_systems):
        n = b.n_atoms(k)
        b.set_positions(k, x[off:off + n])
        off += n
    a.step(5)
    b.step(5)
    for p, q in zip(all_positions(a), all_positions(b)):
        np.testing.assert_array_equal(p, q)


def test_trajectory_capture_matches_positions(origami, tmp_path):
    eng, chains = make_engine(origami)
    path = str(tmp_path / "traj.pdb")
    expect = []
    with origami.Trajectory(chains[1], path, "capture") as t:
        for _ in range(4):
            eng.step(7)
            t.capture(eng, 1)
            expect.append(eng.positions(1))
        t.write(expect[-1])  # a host frame after the captured ones
    lines = open(path).read().splitlines()
    models, cur = [], None
    for l in lines:
        if l.startswith("MODEL"):
            cur = []
        elif l.startswith("ATOM"):
            cur.append([float(l[30:38]), float(l[38:46]), float(l[46:54])])
        elif l.startswith("ENDMDL"):
            models.append(np.array(cur))
    assert len(models) == 5
    for m, x in zip(models, expect + [expect[-1]]):
        assert m.shape == x.shape
        np.testing.assert_allclose(m, x, atol=5.1e-4)
    with pytest.raises(origami.OrigamiError):
        with origami.Trajectory(chains[0], str(tmp_path / "bad.pdb")) as t:
            t.capture(eng, 1)  # system 1 is not chain 0's size
