"""The reference's small configurations run end to end on the GPU and checked
against the FP64 CPU oracle.

C1  one seeded 20-residue chain (xoshiro256++ seed 0), extended NeRF build,
    L-BFGS to gradient RMS < 1 kJ/mol/nm, then 2 000 BAOAB steps at 310 K,
    dt 1 fs, gamma 2 ps^-1, bonded + LJ + Coulomb + GB, no cutoff.  The oracle
    integrates the same start with the same counter-based noise.  Every 100
    steps: the GPU's FP64 energies against the oracle's on the GPU's own
    coordinates (per term < 1e-6 relative), the two trajectories' position
    deviation and potential energies; at the end the GPU forces against the
    oracle's (RMS relative < 1e-5).  The trajectories separate as MD does
    (FP32 pair forces differ from FP64 ones by ~1e-7 relative, and nearby
    trajectories diverge exponentially), so the deviation is reported and
    bounded loosely; the per-frame parity is the tight check.
C2  one seeded 60-residue chain with the analytical PowerSasa term (gamma
    scale 0.25), 10 000 BAOAB steps at 310 K, dt 1 fs, all pairs.  Every 1 000
    steps, per-term energy errors and the force errors (all terms but the
    surface term; the surface term alone) against the oracle on the GPU's
    coordinates.

With OG_REPORT_DIR set, each test writes its numbers there as JSON.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np
import pytest

from conftest import INF, Orc, dp, oracle

pytestmark = pytest.mark.gpu

TERMS = ("bond", "angle", "dihedral", "improper", "lj", "coulomb", "gb", "gb_self", "gb_pair", "total")


def _bench():
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    return bench


def rms_rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


def rel(a, b):
    return abs(a - b) / max(abs(b), 1.0)


def _report(name: str, data: dict) -> None:
    d = os.environ.get("OG_REPORT_DIR")
    if d:
        os.makedirs(d, exist_ok=True)
        with open(os.path.join(d, name), "w") as fh:
            json.dump(data, fh, indent=1)


def _minimised_chain(origami, n_res: int, seed: int, gtol_rms: float, max_steps: int):
    from origami_b200.minimize import MinimizeOptions, minimize_chain
    ch = origami.Chain.build(_bench().seeded_sequence(n_res, seed))
    res = minimize_chain(ch, origami.Params.all_pairs(),
                         MinimizeOptions(max_steps=max_steps, gradient_tol=gtol_rms, gradient_norm="rms"))
    return ch, res


def test_c1_trajectory_and_energy_trace(origami):
    ch, mres = _minimised_chain(origami, 20, 0, 0.1, 20000)
    assert mres.converged, mres
    x0 = ch.positions
    params = origami.Params.all_pairs(dt_fs=1.0, friction_ps_inv=2.0, constrain_h_bonds=False, seed=2024)
    eng = origami.Engine(params)
    eng.add_system(ch, x0, 310.0)
    eng.finalize()
    eng.init_velocities(0, 17, remove_com=True)
    v0 = eng.velocities(0)
    orc = Orc(ch)
    x = np.ascontiguousarray(x0.copy())
    v = np.ascontiguousarray(v0.copy())
    f = orc.total_force(x, INF, INF, INF)
    frames = []
    every, total = 100, 2000
    for k in range(0, total, every):
        eng.step(every)
        fails = oracle().orc_baoab(orc.tp, dp(x), dp(v), dp(f), every, 1.0, 2.0, 310.0, 0, 2024, 0, k,
                                   INF, INF, INF)
        assert fails == 0
        xg = eng.positions(0)
        eg = eng.energies(0)
        ref_same = orc.energy_terms(xg, INF, INF)
        ref_own = orc.energy_terms(x, INF, INF)
        worst = max(rel(eg[t], ref_same[t]) for t in TERMS)
        assert worst < 1e-6, (k + every, {t: (eg[t], ref_same[t]) for t in TERMS})
        frames.append({"step": k + every, "gpu_potential_kj": eg["total"], "oracle_potential_kj": ref_own["total"],
                       "max_term_rel_err_same_coords": worst,
                       "position_rmsd_a": float(np.sqrt(((xg - x) ** 2).sum(1).mean())),
                       "position_max_dev_a": float(np.abs(xg - x).max())})
    xg = eng.positions(0)
    f_gpu = eng.total_force(0)
    f_ref = orc.total_force(xg, INF, INF, INF)
    ferr = rms_rel(f_gpu, f_ref)
    assert ferr < 1e-5, ferr
    st = eng.stats(0)
    assert not st["diverged"]
    # the two runs share noise and start; they separate slowly
    assert frames[0]["position_max_dev_a"] < 1e-3, frames[0]
    e_gpu = np.array([fr["gpu_potential_kj"] for fr in frames[10:]])
    e_orc = np.array([fr["oracle_potential_kj"] for fr in frames[10:]])
    assert abs(e_gpu.mean() - e_orc.mean()) < 3.0 * max(e_orc.std(), 1.0), (e_gpu.mean(), e_orc.mean())
    _report("c1_trajectory.json", {
        "config": "C1: seeded 20-residue chain, L-BFGS to gradient RMS < 0.1 kJ/mol/A, 2000 BAOAB steps, 310 K, "
                  "dt 1 fs, gamma 2 ps^-1, all pairs, no SHAKE; GPU (FP32 pair math, FP64 integrator and "
                  "energies) vs the FP64 oracle with the same noise",
        "atoms": ch.n_atoms, "lbfgs_steps": mres.steps, "lbfgs_final_kj": mres.final_energy,
        "final_force_rms_rel_err": ferr, "frames": frames})


def test_c2_per_term_errors_with_surface_term(origami):
    ch, mres = _minimised_chain(origami, 60, 0, 0.5, 20000)
    x0 = ch.positions
    mk = lambda sasa: origami.Params.all_pairs(dt_fs=1.0, friction_ps_inv=2.0, constrain_h_bonds=False,  # noqa
                                               seed=77, include_sasa=sasa, sasa_gamma_scale=0.25)
    eng = origami.Engine(mk(True))
    eng.add_system(ch, x0, 310.0)
    eng.finalize()
    eng.init_velocities(0, 23, remove_com=True)
    probe = origami.Engine(mk(False))  # the same coordinates without the surface term
    probe.add_system(ch, x0, 310.0)
    probe.finalize()
    orc = Orc(ch)
    o = oracle()
    el = ch.topology().element
    rad = np.array([o.orc_sasa_radius(int(e)) for e in el])
    gam = np.array([o.orc_sasa_gamma(int(e), 0.25) for e in el])
    frames = []
    for k in range(10):
        eng.step(1000)
        x = eng.positions(0)
        eg = eng.energies(0)
        ref = orc.energy_terms(x, INF, INF)
        area = np.zeros(x.shape[0])
        o.orc_sasa_areas(x.shape[0], dp(np.ascontiguousarray(x)), dp(rad), dp(area))
        ref["sasa"] = float((gam * area).sum())
        ref["total"] += ref["sasa"]
        f_all = eng.total_force(0)
        probe.set_positions(0, x)
        f_rest = probe.total_force(0)
        f_rest_ref = orc.total_force(x, INF, INF, INF)
        f_sasa_ref = np.zeros_like(x)
        o.orc_sasa_forces_tangent_one_root(x.shape[0], dp(np.ascontiguousarray(x)), dp(rad), dp(gam),
                                           dp(f_sasa_ref))
        errs = {t: rel(eg[t], ref[t]) for t in TERMS + ("sasa",)}
        fr = {"step": (k + 1) * 1000, "energy_rel_err": errs,
              "energy_kj": {t: eg[t] for t in TERMS + ("sasa",)},
              "force_rms_rel_err_without_surface": rms_rel(f_rest, f_rest_ref),
              "force_rms_rel_err_surface_term": rms_rel(f_all - f_rest, f_sasa_ref),
              "force_rms_rel_err_total": rms_rel(f_all, f_rest_ref + f_sasa_ref)}
        frames.append(fr)
        assert max(errs.values()) < 1e-6, fr
        assert fr["force_rms_rel_err_without_surface"] < 1e-5, fr
        assert fr["force_rms_rel_err_total"] < 1e-5, fr
    st = eng.stats(0)
    assert not st["diverged"]
    worst = {t: max(f["energy_rel_err"][t] for f in frames) for t in TERMS + ("sasa",)}
    _report("c2_per_term_errors.json", {
        "config": "C2: seeded 60-residue chain, L-BFGS-relaxed, 10000 BAOAB steps, 310 K, dt 1 fs, gamma 2 ps^-1, "
                  "all pairs, analytical PowerSasa gamma scale 0.25; GPU energies and forces vs the FP64 oracle "
                  "on the GPU's coordinates every 1000 steps",
        "atoms": ch.n_atoms, "lbfgs_steps": mres.steps,
        "precision": "FP32 pair math with int64 fixed-point force sums; FP64 integrator, Born-integral tile sums, "
                     "energies and PowerSasa",
        "worst_energy_rel_err": worst,
        "worst_force_rms_rel_err": {k: max(f[k] for f in frames) for k in
                                    ("force_rms_rel_err_without_surface", "force_rms_rel_err_surface_term",
                                     "force_rms_rel_err_total")},
        "frames": frames})
