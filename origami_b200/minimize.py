"""L-BFGS energy minimisation on the GPU force/energy boundary.

Host driver restating dynamics/src/lbfgs.rs:61-254 (two-loop recursion,
history of 10 (s, y) pairs, steepest-descent fallback with history reset) and
dynamics/src/line_search.rs:52-101 (backtracking Armijo, alpha0 capped so no
coordinate moves more than max_step_a, contraction 0.5, c1 1e-4).  Every
gradient is an og_compute_forces call and every line-search trial an
og_compute_energies call (FP64 on the device), so the energy the line search
sees is exactly origami's total_energy_with_options (energy_eval.rs:20).

The reference's convergence test is the L-infinity gradient norm in kJ/mol/A;
`gradient_norm="rms"` tests the RMS instead (what the C1 configuration's
"gradient RMS < 1 kJ/mol/nm" asks for: 0.1 kJ/mol/A).
"""
from __future__ import annotations

from collections import deque
from dataclasses import dataclass

import numpy as np


@dataclass
class MinimizeOptions:
    """dynamics/src/minimize.rs:16-38 / lbfgs.rs:23-48."""
    max_steps: int = 500
    gradient_tol: float = 1.0
    energy_tol: float = 0.01
    max_step_a: float = 0.1
    history: int = 10
    alpha0: float = 1.0
    contraction: float = 0.5
    c1: float = 1e-4
    min_alpha: float = 1e-12
    gradient_norm: str = "linf"


@dataclass
class MinimizeResult:
    steps: int
    initial_energy: float
    final_energy: float
    max_force: float
    converged: bool
    line_search_failures: int


def _norm(g: np.ndarray, kind: str) -> float:
    if kind == "rms":
        return float(np.sqrt(np.mean(g * g)))
    return float(np.max(np.abs(g))) if g.size else 0.0


class _System:
    def __init__(self, engine, sys: int):
        self.e, self.s = engine, sys

    def x(self) -> np.ndarray:
        return self.e.positions(self.s).reshape(-1)

    def set_x(self, x: np.ndarray) -> None:
        self.e.set_positions(self.s, x.reshape(-1, 3))

    def energy(self) -> float:
        return self.e.energies(self.s)["total"]

    def grad(self) -> np.ndarray:
        return -self.e.total_force(self.s).reshape(-1)


def _backtracking(sys: _System, x0: np.ndarray, p: np.ndarray, g: np.ndarray, e0: float, alpha0: float,
                  o: MinimizeOptions):
    p_dot_g = float(p @ g)
    if p_dot_g >= 0.0:
        return None
    alpha = alpha0
    while alpha >= o.min_alpha:
        sys.set_x(x0 + alpha * p)
        e_new = sys.energy()
        if e_new <= e0 + o.c1 * alpha * p_dot_g:
            sys.set_x(x0)
            return alpha, e_new
        alpha *= o.contraction
    sys.set_x(x0)
    return None


def _two_loop(g, hs, hy, hr):
    q = g.copy()
    alpha = [0.0] * len(hs)
    for i in range(len(hs) - 1, -1, -1):
        alpha[i] = hr[i] * float(hs[i] @ q)
        q -= alpha[i] * hy[i]
    sy = float(hs[-1] @ hy[-1])
    yy = float(hy[-1] @ hy[-1])
    r = (sy / yy if yy > 0.0 else 1.0) * q
    for i in range(len(hs)):
        beta = hr[i] * float(hy[i] @ r)
        r += (alpha[i] - beta) * hs[i]
    return -r


def lbfgs(engine, sys: int = 0, opts: MinimizeOptions | None = None) -> MinimizeResult:
    """Minimise system `sys` of a finalised Engine in place.

    The reference evaluates the gradient at the top of every iteration and
    the energy before every line search; both were already taken at that
    point (the gradient for the last curvature pair y, the energy by the
    accepted line-search trial).  Device forces and energies are
    deterministic, so those values are reused instead of recomputed -- the
    iterates are the same -- which halves the evaluations per iteration.
    Positions are tracked on the host: the device holds exactly the array
    last set."""
    o = opts or MinimizeOptions()
    S = _System(engine, sys)
    initial = S.energy()
    e_prev = initial
    hs, hy, hr = deque(), deque(), deque()
    failures, steps, converged, max_force = 0, 0, False, float("inf")
    x = S.x()
    g_known, e_known = None, initial
    for step in range(o.max_steps):
        steps = step
        g = g_known if g_known is not None else S.grad()
        g_known = None
        max_force = _norm(g, o.gradient_norm)
        if max_force < o.gradient_tol:
            converged = True
            break
        direction = -g if not hs else _two_loop(g, hs, hy, hr)
        md = float(np.max(np.abs(direction)))
        a0 = min(o.alpha0, o.max_step_a / md) if md > 0 else o.alpha0
        e_now = e_known if e_known is not None else S.energy()
        res = _backtracking(S, x, direction, g, e_now, a0, o)
        if res is None:
            failures += 1
            sd = -g
            md2 = float(np.max(np.abs(sd)))
            a02 = min(o.alpha0, o.max_step_a / md2) if md2 > 0 else o.alpha0
            res2 = _backtracking(S, x, sd, g, e_now, a02, o)
            if res2 is None:
                failures += 1
                break
            x = x + res2[0] * sd
            S.set_x(x)
            hs.clear(); hy.clear(); hr.clear()
            e_prev = e_known = res2[1]
            continue
        alpha, e_new = res
        step_vec = alpha * direction
        x = x + step_vec
        S.set_x(x)
        g_known = S.grad()
        e_known = e_new
        y = g_known - g
        sy = float(step_vec @ y)
        if sy > 1e-12:
            if len(hs) == o.history:
                hs.popleft(); hy.popleft(); hr.popleft()
            hs.append(step_vec); hy.append(y); hr.append(1.0 / sy)
        if abs(e_prev - e_new) < o.energy_tol and max_force < o.gradient_tol:
            converged = True
            steps = step + 1
            break
        e_prev = e_new
    final = e_known if e_known is not None else S.energy()
    return MinimizeResult(steps, initial, final, max_force, converged, failures)


def minimize_chain(chain, params=None, opts: MinimizeOptions | None = None) -> MinimizeResult:
    """geom chain -> one-system engine -> L-BFGS -> positions written back
    (dynamics/src/minimize.rs:76)."""
    from . import Engine, Params
    eng = Engine(params or Params())
    eng.add_system(chain, chain.positions, 0.0)
    eng.finalize()
    res = lbfgs(eng, 0, opts)
    chain.positions = eng.positions(0)
    eng.close()
    return res


class _AllSystems:
    """Every system of an engine as one minimisation problem: the sum of the
    systems' energies over their concatenated coordinates (the systems do
    not interact, so its minimum is each system's minimum).  Positions and
    forces move through the whole-engine state (og_get_state /
    og_set_state), energies through og_compute_energies(sys = -1)."""

    FIXED_SCALE = 2.0 ** 32  # fixed-point force units per kJ/mol/A

    def __init__(self, engine):
        self.e = engine

    def positions(self, _):
        return self.e.get_state(parts=("positions",))["positions"]

    def set_positions(self, _, x):
        self.e.set_state({"positions": np.ascontiguousarray(x, dtype=np.float64).reshape(-1, 3)})

    def energies(self, _):
        return {"total": float(sum(e["total"] for e in self.e.all_energies()))}

    def total_force(self, _):
        self.e.total_force(0)  # evaluates every system
        return self.e.get_state(parts=("forces_fixed",))["forces_fixed"] / self.FIXED_SCALE


def minimize_all(engine, opts: MinimizeOptions | None = None) -> MinimizeResult:
    """L-BFGS over every system of a finalised Engine at once, in place:
    one force evaluation per iteration serves the whole batch."""
    return lbfgs(_AllSystems(engine), 0, opts)
