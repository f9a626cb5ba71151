"""GPU parity of the PowerSasa surface term and the Shrake-Rupley areas
against the CPU oracle (oracle/powersasa.cpp), through the C ABI.

Tolerances (FP64 on both sides; the GPU differs from the oracle only by
fused multiply-adds, device transcendentals and summation order):
  SASA forces     max |dF| < 1e-6 kJ/mol/A (fixed-point 2^-32 per term)
  areas           |dA| < 1e-9 * 4 pi R^2 per atom (analytical)
  Shrake-Rupley   identical dot counts, so identical areas to 1e-12
  energy          |dE| < 1e-9 * max(|E|, 1)

Force parity is checked on generic geometry (jittered builds, random atom
clusters).  Idealised NeRF builds contain exact triple points -- three cap
circles through one point, ~600 of them on the extended Trp-cage -- where
two transitions on a circle coincide and the reference keeps whichever sorts
first by an FP64 angle that ties to the last bit.  Rounding decides that tie
(and so which neighbour the vertex is attributed to), and the area is not
differentiable there; on such builds only areas and energies are compared.

In the tangent band (0 < c_sq <= 1e-9) the engine departs from the reference
on purpose (vertex roots, link_boundary in sasa.cu): its forces there are
checked against central differences of the oracle's surface energy instead.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import Orc, ch2_tangent_cluster, dp, oracle

pytestmark = pytest.mark.gpu

TRP = "NLYIQWLKDGGPSSGRPPPS"


def helix(origami, seq):
    return origami.Chain.build(seq, math.radians(-57.0), math.radians(-47.0), math.pi)


def radii_gamma(chain, scale):
    o = oracle()
    el = np.array(chain.topology().element)
    r = np.array([o.orc_sasa_radius(int(e)) for e in el])
    g = np.array([o.orc_sasa_gamma(int(e), scale) for e in el])
    return r, g


def oracle_sasa_forces(x, r, g):
    x = np.ascontiguousarray(x)
    f = np.zeros_like(x)
    oracle().orc_sasa_forces(x.shape[0], dp(x), dp(r), dp(g), dp(f))
    return f


def oracle_areas(x, r):
    x = np.ascontiguousarray(x)
    a = np.zeros(x.shape[0])
    oracle().orc_sasa_areas(x.shape[0], dp(x), dp(r), dp(a))
    return a


def oracle_sr(x, r, n_dots):
    x = np.ascontiguousarray(x)
    a = np.zeros(x.shape[0])
    oracle().orc_shrake_rupley_areas(x.shape[0], dp(x), dp(r), n_dots, dp(a))
    return a


def engine(origami, chain, x, sasa=True, scale=1.0, params=None):
    p = params or origami.Params()
    p.include_sasa = sasa
    p.sasa_gamma_scale = scale
    eng = origami.Engine(p)
    eng.add_system(chain, x, 310.0)
    eng.finalize()
    return eng


def chains(origami):
    ext = origami.Chain.build(TRP)
    hel = helix(origami, TRP)
    rng = np.random.default_rng(3)
    return [("extended", ext, ext.positions), ("helix", hel, hel.positions),
            ("helix_jitter", hel, hel.positions + rng.normal(scale=0.05, size=hel.positions.shape))]


def generic_chains(origami):
    """Builds with every coordinate perturbed: no exact triple points."""
    rng = np.random.default_rng(11)
    out = []
    for name, ch, x in chains(origami):
        if name.endswith("jitter"):
            out.append((name, ch, x))
        else:
            out.append((name + "_jitter", ch, x + rng.normal(scale=0.02, size=x.shape)))
    return out


def cluster_topology(origami, el):
    n = len(el)
    z = np.zeros(n)
    e2, e3, e4 = (np.zeros((0, k), np.int32) for k in (2, 3, 4))
    return origami.Topology(
        charge=z.copy(), rmin_half=np.ones(n), epsilon=z.copy(), rmin_half_14=np.ones(n), epsilon_14=z.copy(),
        gb_rho=np.full(n, 1.7), gb_scale=np.full(n, 0.72), mass=np.full(n, 12.0),
        element=np.asarray(el, np.int32), bonds=e2, bond_k=np.zeros(0), bond_r0=np.zeros(0), angles=e3,
        angle_k=np.zeros(0), angle_theta0=np.zeros(0), dihedrals=e4, dihedral_term_start=np.zeros(1, np.int32),
        term_k=np.zeros(0), term_n=np.zeros(0, np.int32), term_delta=np.zeros(0), impropers=e4,
        improper_k=np.zeros(0), improper_psi0=np.zeros(0), exclusions=e2, exclusion_kind=np.zeros(0, np.int8),
        constraints=e2, constraint_length=np.zeros(0))


def test_sasa_forces_random_clusters_match_oracle(origami):
    """Many small uncharged clusters of H/C/N/O/S atoms batched as separate
    systems in one engine; only the surface term differs between the engines."""
    rng = np.random.default_rng(2024)
    cases = []
    for _ in range(60):
        n = int(rng.integers(3, 90))
        box = 3.0 + 0.05 * n
        pts = []
        while len(pts) < n:
            p = rng.uniform(-box, box, 3)
            if all(np.linalg.norm(p - q) > 1.1 for q in pts):
                pts.append(p)
        el = rng.choice([0, 1, 1, 2, 3, 5], n)
        el[0] = 1
        cases.append((np.array(pts), el))
    on, off = origami.Params(), origami.Params()
    on.include_sasa = True
    e_on, e_off = origami.Engine(on), origami.Engine(off)
    for x, el in cases:
        t = cluster_topology(origami, el)
        e_on.add_system(t, x)
        e_off.add_system(t, x)
    e_on.finalize()
    e_off.finalize()
    o = oracle()
    for k, (x, el) in enumerate(cases):
        r = np.array([o.orc_sasa_radius(int(e)) for e in el])
        g = np.array([o.orc_sasa_gamma(int(e), 1.0) for e in el])
        f_ref = oracle_sasa_forces(x, r, g)
        df = e_on.total_force(k) - e_off.total_force(k)
        assert np.abs(df - f_ref).max() < 1e-6, k


def dense_shell_cluster(seed, n_shell):
    """A carbon at the origin under a dense half-shell of n_shell atoms
    between 2.4 and 5.4 A on the z > 1 side (at least 0.9 A apart): the
    centre's sphere is cut by every shell atom -- more caps than the default
    kernels hold -- and its other side stays exposed."""
    rng = np.random.default_rng(seed)
    pts = [np.zeros(3)]
    while len(pts) < n_shell + 1:
        d = rng.normal(size=3)
        d[2] = abs(d[2])
        p = d / np.linalg.norm(d) * rng.uniform(2.4, 5.4)
        if p[2] < 1.0:
            continue
        if all(np.linalg.norm(p - q) > 0.9 for q in pts[1:]):
            pts.append(p)
    el = rng.choice([0, 0, 1, 1, 2, 3, 5], n_shell + 1)
    el[0] = 1
    return np.array(pts), el


def test_dense_atoms_beyond_default_capacity_match_oracle(origami):
    """Atoms whose arrangement exceeds the default per-atom capacities (here
    the centre, with 140 caps) are queued for the large-capacity kernels:
    forces, areas and the surface energy still match the oracle, and the
    shell atoms below the limit take the default path in the same launch."""
    x, el = dense_shell_cluster(5, 140)
    r = np.array([oracle().orc_sasa_radius(int(e)) for e in el])
    d = np.linalg.norm(x - x[0], axis=1)
    assert ((d > 0) & (d < r[0] + r)).sum() > 128
    check_cluster(origami, x, el)


def check_cluster(origami, x, el, forces=True):
    """Surface forces (unless forces is False), analytical areas and
    Shrake-Rupley areas of one uncharged cluster against the oracle."""
    o = oracle()
    r = np.array([o.orc_sasa_radius(int(e)) for e in el])
    g = np.array([o.orc_sasa_gamma(int(e), 1.0) for e in el])
    t = cluster_topology(origami, el)
    on, off = origami.Params(), origami.Params()
    on.include_sasa = True
    e_on, e_off = origami.Engine(on), origami.Engine(off)
    e_on.add_system(t, x)
    e_off.add_system(t, x)
    e_on.finalize()
    e_off.finalize()
    if forces:
        df = e_on.total_force(0) - e_off.total_force(0)
        f_ref = oracle_sasa_forces(x, r, g)
        assert np.abs(df - f_ref).max() < 1e-6, np.abs(df - f_ref).max()
    ref = oracle_areas(x, r)
    got = e_off.sasa_areas(0, "powersasa")
    assert np.all(np.abs(got - ref) <= 1e-9 * 4 * math.pi * r**2), np.abs(got - ref).max()
    sr = e_off.sasa_areas(0, "shrake_rupley", 960)
    np.testing.assert_allclose(sr, oracle_sr(x, r, 960), rtol=0, atol=1e-9)


def fibonacci_directions(n):
    k = np.arange(n) + 0.5
    z = 1.0 - 2.0 * k / n
    phi = math.pi * (1.0 + 5.0 ** 0.5) * k
    s = np.sqrt(1.0 - z * z)
    return np.stack([s * np.cos(phi), s * np.sin(phi), z], 1)


def test_many_live_circles_match_oracle(origami):
    """A sulfur under 69 evenly spread hydrogens (75 directions, those near
    the +z pole left out) whose caps on it are all 20 degrees: no cap lies
    inside another, so all 69 circles stay live -- more than the crossing
    masks cover -- each crossing 5 to 9 neighbours, and the caps cover the
    sphere but for one hole at the pole.  The arrangement takes the plain
    pair scan."""
    o = oracle()
    ri, rj, c = o.orc_sasa_radius(5), o.orc_sasa_radius(0), math.cos(math.radians(20.0))
    d = c * ri + math.sqrt((c * ri) ** 2 - (ri * ri - rj * rj))
    dirs = fibonacci_directions(75)
    dirs = dirs[dirs[:, 2] < 0.85]
    assert len(dirs) == 69
    x = np.vstack([np.zeros(3), dirs * d])
    el = np.array([5] + [0] * len(dirs))
    check_cluster(origami, x, el)


def test_tangent_circles_areas_match_oracle(origami):
    """Two caps on a carbon whose circles touch at one point (30-degree
    caps, axes 60 degrees apart: one transition each, by the tangent
    tolerance) and a third cap crossing one of them.  The atom leaves the
    crossing masks for plain counts.  Areas only: the reference's gradient
    divides by the root of c_sq, which vanishes at tangency, so its forces
    there are of order 1e7, with a sign rounding decides (the engine's forces
    in the tangent band are checked against differences of the area in
    test_tangent_band_forces_match_area_differences)."""
    rc = oracle().orc_sasa_radius(1)
    d = rc * math.sqrt(3.0)  # cap cosine d / (2 rc) = cos 30 degrees
    a3 = np.array([math.cos(-0.35), math.sin(-0.35), 0.3])
    dirs = np.array([[1.0, 0.0, 0.0], [math.cos(math.pi / 3), math.sin(math.pi / 3), 0.0], a3 / np.linalg.norm(a3)])
    x = np.vstack([np.zeros(3), dirs * d])
    check_cluster(origami, x, np.array([1, 1, 1, 1]), forces=False)


def test_tangent_band_forces_match_area_differences(origami):
    """In the tangent band a pair has one transition, halfway between its two
    roots, and the reference picks each vertex's root by proximity -- a tie
    that rounding breaks -- so its analytical forces here are of order 1e4
    kJ/mol/A with either sign (MD of CH2 groups meets this whenever the
    H-C-H angle passes twice the cap angle).  The engine gives both vertices
    of the pair the same root, which cancels the 1/sqrt(c_sq) terms: its
    forces match the oracle with the same rule, and central differences of
    the oracle's surface energy."""
    x, el = ch2_tangent_cluster()
    o = oracle()
    r = np.array([o.orc_sasa_radius(int(e)) for e in el])
    g = np.array([o.orc_sasa_gamma(int(e), 1.0) for e in el])
    t = cluster_topology(origami, el)
    on, off = origami.Params(), origami.Params()
    on.include_sasa = True
    e_on, e_off = origami.Engine(on), origami.Engine(off)
    e_on.add_system(t, x)
    e_off.add_system(t, x)
    e_on.finalize()
    e_off.finalize()
    df = e_on.total_force(0) - e_off.total_force(0)

    def energy(xx):
        return float((g * oracle_areas(xx, r)).sum())

    h = 1e-6
    fd = np.zeros_like(x)
    for k in range(len(x)):
        for ax in range(3):
            xp, xm = x.copy(), x.copy()
            xp[k, ax] += h
            xm[k, ax] -= h
            fd[k, ax] = -(energy(xp) - energy(xm)) / (2.0 * h)
    assert np.abs(fd).max() < 1.0
    assert np.abs(df - fd).max() < 1e-3, np.abs(df - fd).max()
    xc = np.ascontiguousarray(x)
    f_rule = np.zeros_like(xc)
    o.orc_sasa_forces_tangent_one_root(len(xc), dp(xc), dp(r), dp(g), dp(f_rule))
    assert np.abs(df - f_rule).max() < 1e-6, np.abs(df - f_rule).max()


@pytest.mark.parametrize("relaxed", [False, True])
def test_sasa_on_the_bench_chain_match_oracle(origami, relaxed):
    """The benchmark's seeded 300-residue chain (4 694 atoms), as built and
    after the bench's relaxation, each coordinate jittered by 0.02 A: surface
    forces at the bench's gamma scale 0.25 and analytical areas against the
    oracle -- the crossing masks, the pair-scan fallback and the
    large-capacity queue at the workload's own size."""
    import os
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    seq, chain = bench.build_workload(origami, 300, 0)
    if relaxed:
        bench.relax(origami, chain, all_pairs=True)
    rng = np.random.default_rng(17)
    x = chain.positions + rng.normal(scale=0.02, size=chain.positions.shape)
    r, g = radii_gamma(chain, 0.25)
    with_s = engine(origami, chain, x, True, 0.25)
    without = engine(origami, chain, x, False)
    df = with_s.total_force(0) - without.total_force(0)
    f_ref = oracle_sasa_forces(x, r, g)
    assert np.abs(df - f_ref).max() < 1e-6, np.abs(df - f_ref).max()
    got = without.sasa_areas(0, "powersasa")
    ref = oracle_areas(x, r)
    assert np.all(np.abs(got - ref) <= 1e-9 * 4 * math.pi * r**2), np.abs(got - ref).max()


@pytest.mark.parametrize("scale", [1.0, 0.25])
def test_sasa_forces_match_oracle(origami, scale):
    for name, ch, x in generic_chains(origami):
        r, g = radii_gamma(ch, scale)
        f_ref = oracle_sasa_forces(x, r, g)
        with_s = engine(origami, ch, x, True, scale)
        without = engine(origami, ch, x, False)
        df = with_s.total_force(0) - without.total_force(0)
        err = np.abs(df - f_ref).max()
        assert err < 1e-6, (name, err, np.abs(f_ref).max())
        assert np.abs(f_ref).max() > 0.01
        # and the total still matches the oracle's total force + SASA
        f_tot = Orc(ch).total_force(x) + f_ref
        rel = np.sqrt(((with_s.total_force(0) - f_tot) ** 2).sum() / (f_tot ** 2).sum())
        assert rel < 1e-5, (name, rel)


def test_powersasa_areas_match_oracle(origami):
    for name, ch, x in chains(origami):
        r, _ = radii_gamma(ch, 1.0)
        ref = oracle_areas(x, r)
        eng = engine(origami, ch, x, False)
        got = eng.sasa_areas(0, "powersasa")
        tol = 1e-9 * 4 * math.pi * r**2
        bad = np.nonzero(np.abs(got - ref) > tol)[0]
        assert bad.size == 0, (name, bad[:5], got[bad[:5]], ref[bad[:5]])


@pytest.mark.parametrize("n_dots", [960, 4096])
def test_shrake_rupley_areas_match_oracle(origami, n_dots):
    for name, ch, x in chains(origami):
        r, _ = radii_gamma(ch, 1.0)
        ref = oracle_sr(x, r, n_dots)
        eng = engine(origami, ch, x, False)
        got = eng.sasa_areas(0, "shrake_rupley", n_dots)
        np.testing.assert_allclose(got, ref, rtol=0, atol=1e-12 * 4 * math.pi * 3.2**2)


@pytest.mark.parametrize("scale", [1.0, 0.25])
def test_sasa_energy_matches_oracle(origami, scale):
    for name, ch, x in chains(origami):
        r, g = radii_gamma(ch, scale)
        e_ref = float((g * oracle_areas(x, r)).sum())
        eng = engine(origami, ch, x, True, scale)
        en = eng.energies(0)
        assert abs(en["sasa"] - e_ref) <= 1e-9 * max(abs(e_ref), 1.0), (name, en["sasa"], e_ref)
        base = engine(origami, ch, x, False).energies(0)
        assert abs(en["total"] - (base["total"] + en["sasa"])) < 1e-9 * abs(base["total"])


def test_sasa_batched_systems_match_single(origami):
    rows = chains(origami)
    big = origami.Chain.build("ARNDCQEGHILKMFPSTWYV" * 2)
    rows.append(("40-mer", big, big.positions))
    p = origami.Params()
    p.include_sasa = True
    eng = origami.Engine(p)
    for _, ch, x in rows:
        eng.add_system(ch, x, 310.0)
    eng.finalize()
    for k, (name, ch, x) in enumerate(rows):
        single = engine(origami, ch, x, True)
        np.testing.assert_array_equal(eng.total_force(k), single.total_force(0), err_msg=name)
        assert eng.energies(k)["sasa"] == single.energies(0)["sasa"]


def test_sasa_forces_deterministic(origami):
    ch = helix(origami, TRP)
    x = ch.positions
    a = engine(origami, ch, x, True).total_force(0)
    b = engine(origami, ch, x, True).total_force(0)
    assert np.array_equal(a, b)


def test_sasa_md_runs_and_conserves_shape(origami):
    """A short BAOAB run with the surface term stays finite and reports no
    capacity overflow (the step would return an error)."""
    from test_gpu_parity import minimized
    ch = minimized(origami, TRP)
    p = origami.Params(dt_fs=2.0, constrain_h_bonds=True, seed=5)
    p.include_sasa = True
    p.sasa_gamma_scale = 0.25
    eng = origami.Engine(p)
    eng.add_system(ch, ch.positions, 310.0)
    eng.finalize()
    eng.init_velocities(0, 11, True)
    eng.step(200)
    x = eng.positions(0)
    assert np.isfinite(x).all()
    assert eng.energies(0)["sasa"] > 0.0
