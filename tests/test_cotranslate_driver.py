"""Host logic of the co-translation driver (origami_b200/cotranslate.py) on
the CPU: the engines are stand-ins that record what the driver asks of
them, the chain and the velocity stream are the real ones.  With
grow_in_place the run holds one minimisation engine and one dynamics engine,
grows each by exactly the atoms emitted since it last saw the chain (the
dynamics engine with the new atoms' seeded velocities), hands them the whole
chain's positions, and keeps the step count on the dynamics engine; without
it, every minimisation and every slice gets an engine of its own
(run_cotranslate, cotranslate.rs:174-313).
"""
from __future__ import annotations

import numpy as np
import pytest

import origami_b200 as og
import origami_b200.cotranslate as ct
import origami_b200.minimize as mn


class FakeEngine:
    made: list = []

    def __init__(self, params=None):
        self.params = params
        self.x = None
        self.v = None
        self.steps = 0
        self.appends = []
        self.closed = False
        FakeEngine.made.append(self)

    def add_system(self, chain, xyz, temperature_k=310.0):
        self.x = np.array(xyz, dtype=np.float64).reshape(-1, 3)
        self.v = np.zeros_like(self.x)
        return 0

    def finalize(self):
        return self

    def n_atoms(self, sys=0):
        return self.x.shape[0]

    def append_atoms(self, sys, grown, xyz_new, v_new=None):
        xyz_new = np.asarray(xyz_new).reshape(-1, 3)
        assert self.x.shape[0] + xyz_new.shape[0] == grown.n_atoms
        self.appends.append((xyz_new.copy(), None if v_new is None else np.array(v_new)))
        self.x = np.vstack([self.x, xyz_new])
        self.v = np.vstack([self.v, np.zeros_like(xyz_new) if v_new is None else np.asarray(v_new)])

    def set_positions(self, sys, xyz):
        x = np.asarray(xyz).reshape(-1, 3)
        assert x.shape == self.x.shape
        self.x = x.copy()

    def positions(self, sys=0):
        return self.x.copy()

    def velocities(self, sys=0):
        return self.v.copy()

    def set_state(self, state):
        if state.get("velocities") is not None:
            self.v = np.array(state["velocities"])
        if state.get("steps") is not None:
            self.steps = int(state["steps"][0])

    def step(self, n, check=True):
        self.steps += n
        self.x = self.x + 0.001 * n  # a deterministic drift the driver must carry over
        self.v = self.v * 0.5
        return 0

    def close(self):
        self.closed = True


def fake_lbfgs(engine, sys=0, opts=None):
    engine.set_positions(sys, engine.positions(sys) - 0.0005)  # a deterministic "minimisation"
    return mn.MinimizeResult(3, 1.0, 0.5, 0.1, True, 0)


@pytest.fixture
def fakes(monkeypatch):
    FakeEngine.made = []
    monkeypatch.setattr(ct, "Engine", FakeEngine)
    monkeypatch.setattr(og, "Engine", FakeEngine)  # minimize_chain's engine
    monkeypatch.setattr(ct, "lbfgs", fake_lbfgs)
    monkeypatch.setattr(mn, "lbfgs", fake_lbfgs)
    return FakeEngine


def _run(grow):
    opts = og.LangevinOptions(dt_fs=1.0, temperature_k=300.0, save_every=0, seed=3)
    t = ct.CotranslateTimings()
    chain = ct.run_cotranslate(ct.UniformRibosome("GAVLK", 10.0), opts, 5, None, params=og.Params(), timings=t,
                               grow_in_place=grow)
    return chain, t


def test_grow_in_place_keeps_two_engines_and_appends_only_new_atoms(fakes):
    chain, t = _run(True)
    assert len(fakes.made) == 2
    mins = [e for e in fakes.made if not e.params.include_sasa and e.params.dt_fs == 1.0 and e.params.seed == 0]
    dyn = [e for e in fakes.made if e.params.seed == 3]
    assert len(mins) == 1 and len(dyn) == 1
    m, d = mins[0], dyn[0]
    assert all(e.closed for e in fakes.made)
    # the minimisation engine grew once per residue after the first, the
    # dynamics engine once per slice after the first
    assert len(m.appends) == 4 and len(d.appends) == 4
    sizes = [og.Chain.build("GAVLK"[:k]).n_atoms for k in range(1, 6)]
    assert [a[0].shape[0] for a in m.appends] == list(np.diff(sizes))
    assert [a[0].shape[0] for a in d.appends] == list(np.diff(sizes))
    assert all(a[1] is None for a in m.appends) and all(a[1] is not None for a in d.appends)
    # steps: 10 per emission interval, then the 5-step tail, all on one engine
    assert d.steps == 4 * 10 + 5 and t.steps == 45 and t.slices == 5
    assert t.minimize_iterations == 5 * 3
    assert chain.n_atoms == sizes[-1]
    np.testing.assert_allclose(chain.positions, d.x)


def test_grown_and_rebuilt_drivers_agree(fakes):
    a, ta = _run(True)
    n_grown = len(fakes.made)
    fakes.made.clear()
    b, tb = _run(False)
    assert n_grown == 2 and len(fakes.made) == 10  # a minimisation and a slice engine per residue
    assert ta.steps == tb.steps and ta.slices == tb.slices
    np.testing.assert_allclose(a.positions, b.positions, rtol=0, atol=1e-12)


def test_new_atoms_get_the_seeded_velocities(fakes):
    """The dynamics engine receives, for each new atom, the draw that
    seed_new_atom_velocities makes from the run's xoshiro stream."""
    _run(True)
    d = [e for e in fakes.made if e.params.seed == 3][0]
    rng = og.Xoshiro256pp(3)
    ch = og.Chain.build("G")
    v = ct.seed_new_atom_velocities(ch, np.zeros((0, 3)), 300.0, rng)
    for k, aa in enumerate("AVLK"):
        ch.append(aa)
        n_old = v.shape[0]
        v = ct.seed_new_atom_velocities(ch, v, 300.0, rng)
        np.testing.assert_array_equal(d.appends[k][1], v[n_old:])
