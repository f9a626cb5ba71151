"""Co-translational chain growth on the GPU (dynamics/src/cotranslate.rs).

The driver alternates, as run_cotranslate (cotranslate.rs:174-313) does,
between emitting the next residue -- appended with origami's NeRF builder,
relieved by a short L-BFGS, new atoms seeded with Maxwell-Boltzmann
velocities from the run's xoshiro stream (langevin.rs:417-447) -- and a
BAOAB slice up to the next emission time (run_slice, cotranslate.rs:315-384:
no SHAKE, the ribosome's exit tunnel as an external force, reference
cutoffs).  A tail slice of tail_steps follows the last residue.

The reference rebuilds its ForceScratch -- an O(N^2) exclusion matrix
among it -- for every slice (cotranslate.rs:318-319, scratch.rs:233-251).
Here the run keeps two engines for its whole length, one for the per-append
L-BFGS and one for the slices, and grows both in place when a residue is
emitted (og_engine_append_atoms): only the new atoms' parameters, positions
and velocities, their exclusion-mask blocks, bonded terms and SHAKE
clusters go to the device, and the old atoms' velocities and the step count
never leave it.  `grow_in_place=False` instead builds a fresh engine for
every slice and every minimisation (tables in O(atoms), tile work lists in
O(tiles^2)); both give the same trajectory.  The engine's O-step noise is
keyed by the run's global step count, so no slice repeats another's noise.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import (BOLTZMANN_KJ_PER_MOL_K, Chain, Engine, LangevinOptions, Params, Xoshiro256pp, _check, _dptr, lib)
from .minimize import MinimizeOptions, lbfgs, minimize_chain

ACCEL_FACTOR = 1.0e-4  # langevin.rs ACCEL_FACTOR: kJ/mol/A/Da -> A/fs^2


@dataclass
class UniformRibosome:
    """Residue i is emitted at i * interval_fs (cotranslate.rs:64-88)."""
    sequence: str
    interval_fs: float

    def emission_time_fs(self, residue_idx: int) -> float:
        return residue_idx * max(self.interval_fs, 0.0)


@dataclass
class CylindricalTunnel:
    """Soft exit-tunnel confinement (cotranslate.rs:100-154); defaults as
    CylindricalTunnel::default."""
    axis_origin: tuple = (0.0, 0.0, 0.0)
    axis_direction: tuple = (0.0, 0.0, 1.0)
    radius_a: float = 12.0
    length_a: float = 80.0
    k_confine: float = 50.0

    def apply_to(self, engine: Engine) -> None:
        o = np.ascontiguousarray(self.axis_origin, dtype=np.float64)
        d = np.ascontiguousarray(self.axis_direction, dtype=np.float64)
        _check(lib().og_set_tunnel(engine._h, _dptr(o), _dptr(d), float(self.radius_a), float(self.length_a),
                                   float(self.k_confine)))


@dataclass
class CotranslateFrame:
    """cotranslate.rs:158-163."""
    time_fs: float
    residue_count: int
    positions: np.ndarray
    instantaneous_temperature_k: float


# minimize after every append (cotranslate.rs:218-231)
APPEND_MINIMIZE = MinimizeOptions(max_steps=200, gradient_tol=10.0, energy_tol=0.1, max_step_a=0.1)


def seed_new_atom_velocities(chain: Chain, velocities: np.ndarray, temperature_k: float,
                             rng: Xoshiro256pp) -> np.ndarray:
    """Existing atoms keep their velocities; atoms added since get
    sigma * gaussian per component, sigma = sqrt(kB T ACCEL / m), drawn x, y,
    z per atom in atom order (langevin.rs:417-447)."""
    n = chain.n_atoms
    old = velocities.shape[0]
    if n <= old:
        return velocities
    mass = chain.topology().mass
    kbt = BOLTZMANN_KJ_PER_MOL_K * temperature_k
    out = np.empty((n, 3))
    out[:old] = velocities
    for i in range(old, n):
        sigma = math.sqrt(kbt * ACCEL_FACTOR / mass[i])
        out[i] = [sigma * rng.gaussian(), sigma * rng.gaussian(), sigma * rng.gaussian()]
    return out


def _temperature(velocities: np.ndarray, mass: np.ndarray) -> float:
    ke = 0.5 * float((mass[:, None] * velocities * velocities).sum()) / ACCEL_FACTOR
    dof = 3.0 * velocities.shape[0]
    return 2.0 * ke / (dof * BOLTZMANN_KJ_PER_MOL_K) if dof > 0 else 0.0


class CotranslateDiverged(RuntimeError):
    """A slice diverged; residue_count and time_fs say where, positions and
    velocities hold the slice's starting state."""

    def __init__(self, residue_count: int, time_fs: float, message: str, positions=None, velocities=None):
        super().__init__(f"slice after residue {residue_count} (t = {time_fs:.0f} fs) diverged: {message}")
        self.residue_count = residue_count
        self.time_fs = time_fs
        self.positions = positions
        self.velocities = velocities


@dataclass
class CotranslateTimings:
    """Wall time of a run by part (seconds): the per-residue L-BFGS (and its
    iterations), engine construction or growth (tables, tile lists, graph),
    and the dynamics slices."""
    minimize_s: float = 0.0
    minimize_iterations: int = 0
    build_s: float = 0.0
    steps_s: float = 0.0
    steps: int = 0
    slices: int = 0
    # learned radii: plain-GB judgements made, slices that ended with the
    # network still in use, and the largest error a slice's last judgement saw
    judges: int = 0
    learned_slices: int = 0
    judge_max_error: float = -1.0


def run_cotranslate(ribosome, opts: LangevinOptions, tail_steps: int, external: CylindricalTunnel | None = None,
                    callback=None, params: Params | None = None, lgb_params=None, judge_interval: int = 0,
                    timings: CotranslateTimings | None = None, deadline: float | None = None,
                    grow_in_place: bool = True) -> Chain | None:
    """Grows the ribosome's sequence residue by residue with dynamics in
    between (cotranslate.rs:174-313); returns the final chain (None for an
    empty sequence).  callback(CotranslateFrame) receives every save_every-th
    step of each slice, and the emission moment of a slice with no steps.
    params.born_mode = 1 runs the slices with learned Born radii from
    lgb_params (the network's parameter vector), judged by plain GB every
    judge_interval steps; opts.constrain_h_bonds puts SHAKE on the slices
    (the reference's run_slice has none).  `timings` collects where the wall
    time went; with a deadline (time.perf_counter() value) the growth stops
    after the residue during which it passes.  grow_in_place keeps one
    minimisation engine and one dynamics engine for the whole run and grows
    them per residue; False builds fresh ones every time."""
    seq = ribosome.sequence
    if not seq:
        return None
    base = params or Params()
    if base.born_mode == 1 and lgb_params is None:
        raise ValueError("learned radii need the network's parameters")
    rng = Xoshiro256pp(opts.seed)
    chain: Chain | None = None
    velocities = np.zeros((0, 3))
    clock_fs = 0.0
    steps_done = 0
    grown = _GrowingEngines(opts, external, base, lgb_params, judge_interval) if grow_in_place else None
    try:
        for i, aa in enumerate(seq):
            if deadline is not None and time.perf_counter() > deadline:
                break
            clock_fs = max(clock_fs, ribosome.emission_time_fs(i))
            if chain is None:
                chain = Chain.build(aa)
            else:
                chain.append(aa)
            t0 = time.perf_counter()
            if grown is not None:
                mres = grown.minimize(chain)
            else:
                mres = minimize_chain(chain, params=_minimize_params(base), opts=APPEND_MINIMIZE)
            if timings is not None:
                timings.minimize_s += time.perf_counter() - t0
                timings.minimize_iterations += mres.steps
            velocities = seed_new_atom_velocities(chain, velocities, opts.temperature_k, rng)
            target = ribosome.emission_time_fs(i + 1) if i + 1 < len(seq) else clock_fs + tail_steps * opts.dt_fs
            n_steps = int(round(max(target - clock_fs, 0.0) / opts.dt_fs))
            if n_steps == 0:
                if callback:
                    callback(CotranslateFrame(clock_fs, i + 1, chain.positions,
                                              _temperature(velocities, chain.topology().mass)))
                continue
            if grown is not None:
                t1 = time.perf_counter()
                eng = grown.dynamics(chain, velocities, steps_done)
                if timings is not None:
                    timings.build_s += time.perf_counter() - t1
                velocities = _step_slice(eng, chain, velocities, opts, n_steps, clock_fs, i + 1, callback, timings,
                                         learned=base.born_mode == 1, cumulative_judges=True)
                clock_fs, steps_done = clock_fs + n_steps * opts.dt_fs, steps_done + n_steps
            else:
                clock_fs, steps_done, velocities = _run_slice(chain, velocities, opts, n_steps, external, base,
                                                              clock_fs, steps_done, i + 1, callback, lgb_params,
                                                              judge_interval, timings)
    finally:
        if grown is not None:
            grown.close()
    return chain


def _minimize_params(base: Params) -> Params:
    return Params(nb_cutoff=base.nb_cutoff, born_cutoff=base.born_cutoff, gb_force_cutoff=base.gb_force_cutoff)


def _slice_params(opts: LangevinOptions, base: Params) -> Params:
    return Params(nb_cutoff=base.nb_cutoff, born_cutoff=base.born_cutoff, gb_force_cutoff=base.gb_force_cutoff,
                  dt_fs=opts.dt_fs, friction_ps_inv=opts.friction_ps_inv, constrain_h_bonds=opts.constrain_h_bonds,
                  include_sasa=opts.include_sasa, sasa_gamma_scale=base.sasa_gamma_scale, seed=opts.seed,
                  born_mode=base.born_mode)


def _new_slice_engine(chain: Chain, velocities: np.ndarray, opts: LangevinOptions, external, base: Params,
                      steps_done: int, lgb_params, judge_interval: int) -> Engine:
    eng = Engine(_slice_params(opts, base))
    try:
        eng.add_system(chain, chain.positions, opts.temperature_k)
        eng.finalize()
        if external is not None:
            external.apply_to(eng)
        if base.born_mode == 1:
            from . import lgb
            lgb.set_params(eng, lgb_params)
            lgb.set_judge(eng, judge_interval, 1e-3)
        eng.set_state({"velocities": np.ascontiguousarray(velocities, dtype=np.float64),
                       "steps": np.array([steps_done], dtype=np.int64)})
    except Exception:
        eng.close()
        raise
    return eng


class _GrowingEngines:
    """The run's two engines, built for the first residue and grown in place
    for each one after it (og_engine_append_atoms): the minimisation engine
    (reference cutoffs, no surface term) and the dynamics engine (the run's
    options, tunnel and learned radii set once).  The dynamics engine keeps
    its velocities and step count on the device between slices; with learned
    radii the judge counts its interval over the whole run, and a fallback
    to plain GB lasts for the rest of it."""

    def __init__(self, opts: LangevinOptions, external, base: Params, lgb_params, judge_interval: int):
        self.opts, self.external, self.base = opts, external, base
        self.lgb_params, self.judge_interval = lgb_params, judge_interval
        self.min_eng: Engine | None = None
        self.dyn_eng: Engine | None = None

    def close(self) -> None:
        for eng in (self.min_eng, self.dyn_eng):
            if eng is not None:
                eng.close()
        self.min_eng = self.dyn_eng = None

    @staticmethod
    def _grow(eng: Engine, chain: Chain, velocities: np.ndarray | None = None) -> None:
        x = chain.positions
        n_old = eng.n_atoms(0)
        if x.shape[0] > n_old:
            eng.append_atoms(0, chain, x[n_old:], None if velocities is None else velocities[n_old:])
        eng.set_positions(0, x)

    def minimize(self, chain: Chain):
        """L-BFGS after an append (cotranslate.rs:218-231), in place."""
        if self.min_eng is None:
            self.min_eng = Engine(_minimize_params(self.base))
            self.min_eng.add_system(chain, chain.positions, 0.0)
            self.min_eng.finalize()
        else:
            self._grow(self.min_eng, chain)
        res = lbfgs(self.min_eng, 0, APPEND_MINIMIZE)
        chain.positions = self.min_eng.positions(0)
        return res

    def dynamics(self, chain: Chain, velocities: np.ndarray, steps_done: int) -> Engine:
        """The dynamics engine holding the chain as it is now: the atoms
        emitted since the last slice appended with their seeded velocities,
        every position from the minimisation."""
        if self.dyn_eng is None:
            self.dyn_eng = _new_slice_engine(chain, velocities, self.opts, self.external, self.base, steps_done,
                                             self.lgb_params, self.judge_interval)
        else:
            self._grow(self.dyn_eng, chain, velocities)
        return self.dyn_eng


def _step_slice(eng: Engine, chain: Chain, velocities: np.ndarray, opts: LangevinOptions, n_steps: int,
                clock_fs: float, residue_count: int, callback, timings: CotranslateTimings | None,
                learned: bool = False, cumulative_judges: bool = False) -> np.ndarray:
    """n_steps BAOAB steps in save_every chunks (run_slice, cotranslate.rs:
    346-384); the chain takes the final positions, the velocities are
    returned.  With learned radii the judge's record goes to `timings`
    (its judgement count is the engine's running total when
    cumulative_judges)."""
    t1 = time.perf_counter()
    chunk = opts.save_every if opts.save_every > 0 else n_steps
    done = 0
    while done < n_steps:
        k = min(chunk, n_steps - done)
        st = eng.step(k, check=False)
        if st != 0:
            raise CotranslateDiverged(residue_count, clock_fs + (done + k) * opts.dt_fs,
                                      lib().og_last_error().decode(), chain.positions,
                                      np.ascontiguousarray(velocities, dtype=np.float64))
        done += k
        if callback and opts.save_every > 0 and done % opts.save_every == 0:
            _, t_inst = eng.kinetic(0)
            callback(CotranslateFrame(clock_fs + done * opts.dt_fs, residue_count, eng.positions(0), t_inst))
    chain.positions = eng.positions(0)
    velocities = eng.velocities(0)
    if timings is not None:
        timings.steps_s += time.perf_counter() - t1
        timings.steps += n_steps
        timings.slices += 1
        if learned:
            from . import lgb
            st = lgb.status(eng)
            timings.judges = st["judged"] + (0 if cumulative_judges else timings.judges)
            timings.learned_slices += int(st["active"])
            timings.judge_max_error = max(timings.judge_max_error, st["last_error"])
    return velocities


def _run_slice(chain: Chain, velocities: np.ndarray, opts: LangevinOptions, n_steps: int,
               external: CylindricalTunnel | None, base: Params, clock_fs: float, steps_done: int,
               residue_count: int, callback, lgb_params=None, judge_interval: int = 0,
               timings: CotranslateTimings | None = None):
    """One slice in an engine built for it (the grow_in_place=False path)."""
    t0 = time.perf_counter()
    eng = _new_slice_engine(chain, velocities, opts, external, base, steps_done, lgb_params, judge_interval)
    try:
        if timings is not None:
            timings.build_s += time.perf_counter() - t0
        velocities = _step_slice(eng, chain, velocities, opts, n_steps, clock_fs, residue_count, callback, timings,
                                 learned=base.born_mode == 1)
    finally:
        eng.close()
    return clock_fs + n_steps * opts.dt_fs, steps_done + n_steps, velocities
