"""Pins the CPU oracle (the checker of every GPU parity test) to origami's
known answers and its own invariants: the Coulomb constant, finite-difference
gradients of every term (the reference's main correctness tool, ε = 1e-5),
Newton's third law, the xoshiro256++ stream.  The whole-structure energy
pins (extended and native Trp-cage, chignolin, villin) are in
tests/test_host_oracle.py.  CPU only."""
from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import Orc, dp, known, oracle

TRP_CAGE = "NLYIQWLKDGGPSSGRPPPS"


def test_coulomb_known_value():
    # energy/src/nonbonded.rs known_coulomb_value: +1e and -1e at 5 A
    assert abs(-332.0637 / 5.0 * 4.184 - known("coulomb_unit_pair_5A_kj")) < 0.01


def test_born_radii_floor(origami):
    # With origami's descreening formula (gb.rs:347-369) every pair term is
    # negative for these geometries, so each radius clamps to rho - 0.09.
    ch = origami.Chain.build(TRP_CAGE)
    orc = Orc(ch)
    r = orc.born_radii()
    t = ch.topology()
    assert np.allclose(r, t.gb_rho - 0.09, rtol=0, atol=0)


def _bump_energy(orc, x, i, axis, eps, fn):
    xp = x.copy(); xp[i, axis] += eps
    xm = x.copy(); xm[i, axis] -= eps
    return -(fn(xp) - fn(xm)) / (2 * eps)


def test_bonded_force_finite_difference(origami):
    # energy/src/forces_bonded.rs tests (tol 1e-2 bonds, 1e-1 angles/dihedrals/impropers)
    ch = origami.Chain.build("NAKW")
    orc = Orc(ch)
    x = ch.positions
    # perturb the geometry away from the build so every term has a gradient
    rng = np.random.default_rng(1)
    x = x + rng.normal(scale=0.05, size=x.shape)
    f = orc.bonded_force(x)
    e = np.zeros(4)

    def energy(xx):
        xx = np.ascontiguousarray(xx)
        oracle().orc_bonded_energy(orc.tp, dp(xx), dp(e))
        return e.sum()

    for i in range(0, ch.n_atoms, 3):
        for a in range(3):
            num = _bump_energy(orc, x, i, a, 1e-5, energy)
            assert abs(num - f[i, a]) < 1e-1 + 1e-4 * abs(num), (i, a, num, f[i, a])
    assert np.linalg.norm(f.sum(axis=0)) < 1e-6  # Newton's third law (forces_bonded.rs:504-525)


def test_total_force_finite_difference(origami):
    # energy/src/forces.rs total_force_finite_difference: frozen Born radii,
    # GB pair energy within the same 10 A cutoff the force uses (tol 1.0).
    ch = origami.Chain.build("KAE")
    orc = Orc(ch)
    x = ch.positions
    t = ch.topology()
    f = orc.total_force(x)
    R = orc.born_radii(x)
    q = t.charge
    pref = -0.5 * (1 - 1 / 78.5) * 332.0637 * 4.184
    e_b = np.zeros(4)
    e_nb = np.zeros(2)

    def energy(xx):
        xx = np.ascontiguousarray(xx)
        oracle().orc_bonded_energy(orc.tp, dp(xx), dp(e_b))
        oracle().orc_nonbonded_energy(orc.tp, dp(xx), 10.0, dp(e_nb))
        d2 = ((xx[:, None] - xx[None]) ** 2).sum(-1)
        iu = np.triu_indices(len(xx), 1)
        rp = R[iu[0]] * R[iu[1]]
        fgb = np.sqrt(d2[iu] + rp * np.exp(-d2[iu] / (4 * rp)))
        m = d2[iu] <= 100.0
        pair = (2 * pref * q[iu[0]] * q[iu[1]] / fgb)[m].sum()
        return e_b.sum() + e_nb.sum() + pair + (pref * q * q / R).sum()

    for i in range(0, 15):
        for a in range(3):
            num = _bump_energy(orc, x, i, a, 1e-5, energy)
            assert abs(num - f[i, a]) < 1.0, (i, a, num, f[i, a])


def test_all_pairs_force_is_gradient(origami):
    # No-cutoff mode: force = -grad(bonded + LJ + bare Coulomb + GB pair) at frozen radii.
    ch = origami.Chain.build("DKWAG")
    orc = Orc(ch)
    x = ch.positions + np.random.default_rng(3).normal(scale=0.02, size=(ch.n_atoms, 3))
    t = ch.topology()
    inf = 1e300
    f = orc.total_force(x, inf, inf, inf)
    R = orc.born_radii(x, inf)
    q = t.charge
    pref = -0.5 * (1 - 1 / 78.5) * 332.0637 * 4.184
    e_b, e_nb = np.zeros(4), np.zeros(2)

    def energy(xx):
        xx = np.ascontiguousarray(xx)
        oracle().orc_bonded_energy(orc.tp, dp(xx), dp(e_b))
        oracle().orc_nonbonded_energy(orc.tp, dp(xx), inf, dp(e_nb))
        d2 = ((xx[:, None] - xx[None]) ** 2).sum(-1)
        iu = np.triu_indices(len(xx), 1)
        rp = R[iu[0]] * R[iu[1]]
        fgb = np.sqrt(d2[iu] + rp * np.exp(-d2[iu] / (4 * rp)))
        return e_b.sum() + e_nb.sum() + (2 * pref * q[iu[0]] * q[iu[1]] / fgb).sum()

    worst = 0.0
    for i in range(0, ch.n_atoms, 4):
        for a in range(3):
            num = _bump_energy(orc, x, i, a, 1e-5, energy)
            worst = max(worst, abs(num - f[i, a]) / (1.0 + abs(num)))
    assert worst < 1e-4
    assert np.linalg.norm(f.sum(axis=0)) < 1e-6


def test_xoshiro_stream_matches_reference_recipe(origami):
    # rng.rs: SplitMix64 seeding, xoshiro256++ output, 53-bit uniforms; the
    # Python driver's copy and the oracle's C copy agree bit for bit.
    import ctypes as C
    o = oracle()
    size = o.orc_xoshiro_size()
    buf = C.create_string_buffer(size)
    o.orc_xoshiro_seed.argtypes = [C.c_void_p, C.c_uint64]
    o.orc_xoshiro_u64.argtypes = [C.c_void_p]
    o.orc_xoshiro_u64.restype = C.c_uint64
    o.orc_xoshiro_gaussian.argtypes = [C.c_void_p]
    o.orc_xoshiro_gaussian.restype = C.c_double
    for seed in (0, 42, 0xDEADBEEF, 2 ** 63 + 5):
        o.orc_xoshiro_seed(buf, seed)
        py = origami.Xoshiro256pp(seed)
        for _ in range(50):
            assert o.orc_xoshiro_u64(buf) == py.next_u64()
        o.orc_xoshiro_seed(buf, seed)
        py = origami.Xoshiro256pp(seed)
        for _ in range(20):
            assert o.orc_xoshiro_gaussian(buf) == py.gaussian()
    # moments (rng.rs tests): mean ~0, variance ~1
    g = origami.Xoshiro256pp(7)
    s = np.array([g.gaussian() for _ in range(20000)])
    assert abs(s.mean()) < 0.03 and abs(s.var() - 1) < 0.05


def test_engine_normals_moments():
    o = oracle()
    out = np.zeros(3)
    vals = []
    for atom in range(2000):
        o.orc_engine_normals(123, 0, 7, atom, dp(out))
        vals.append(out.copy())
    v = np.array(vals)
    assert np.all(np.abs(v.mean(0)) < 0.08) and np.all(np.abs(v.var(0) - 1) < 0.1)
    o.orc_engine_normals(123, 0, 7, 5, dp(out))
    a = out.copy()
    o.orc_engine_normals(123, 0, 8, 5, dp(out))
    assert not np.allclose(a, out)


def test_shake_settles_to_target(origami):
    # dynamics/src/shake.rs tests: after one SHAKE call every X-H bond is within tol
    ch = origami.Chain.build("AKS")
    t = ch.topology()
    x0 = ch.positions
    x = x0 + np.random.default_rng(0).normal(scale=0.01, size=x0.shape)
    inv_m = 1.0 / t.mass
    cons = np.ascontiguousarray(t.constraints.astype(np.int32))
    import ctypes as C
    it = oracle().orc_shake(dp(x), dp(np.ascontiguousarray(x0)), dp(inv_m), len(cons),
                            cons.ctypes.data_as(C.POINTER(C.c_int32)), dp(t.constraint_length), 1e-6, 64)
    assert it > 0
    d2 = ((x[cons[:, 0]] - x[cons[:, 1]]) ** 2).sum(1)
    assert np.all(np.abs(d2 - t.constraint_length ** 2) < 1e-6)
