"""Co-translation host logic on the CPU: the ribosome's emission schedule
(cotranslate.rs tests: uniform_ribosome_emission_times), the oracle's tunnel
against the reference's own tunnel tests, and new-atom velocity seeding
from origami's xoshiro stream (langevin.rs:417-447)."""
from __future__ import annotations

import math
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))

import cotranslate as oracle_tunnel  # noqa: E402


def test_uniform_ribosome_emission_times():
    from origami_b200.cotranslate import UniformRibosome
    r = UniformRibosome("AGS", 500.0)
    assert [r.emission_time_fs(i) for i in range(3)] == [0.0, 500.0, 1000.0]
    assert UniformRibosome("A", -5.0).emission_time_fs(3) == 0.0  # interval clamped at 0


def test_oracle_tunnel_matches_reference_tests():
    # cylindrical_tunnel_pushes_atoms_inward
    f = oracle_tunnel.tunnel_forces([[6.0, 0.0, 25.0]], (0, 0, 0), (0, 0, 1), 5.0, 50.0, 10.0)
    np.testing.assert_allclose(f[0], [-10.0, 0.0, 0.0], atol=1e-12)
    # cylindrical_tunnel_no_force_inside (default tunnel)
    f = oracle_tunnel.tunnel_forces([[2.0, 0.0, 40.0]], (0, 0, 0), (0, 0, 1), 12.0, 80.0, 50.0)
    assert (f == 0.0).all()
    # outside the axial extent: no force
    f = oracle_tunnel.tunnel_forces([[30.0, 0.0, -1.0], [30.0, 0.0, 81.0]], (0, 0, 0), (0, 0, 1), 12.0, 80.0, 50.0)
    assert (f == 0.0).all()


def test_new_atom_velocities_follow_the_stream(origami):
    from origami_b200.cotranslate import seed_new_atom_velocities
    ch = origami.Chain.build("A")
    rng = origami.Xoshiro256pp(7)
    v = seed_new_atom_velocities(ch, np.zeros((0, 3)), 310.0, rng)
    n1 = ch.n_atoms
    ch.append("G")
    v2 = seed_new_atom_velocities(ch, v, 310.0, rng)
    np.testing.assert_array_equal(v2[:n1], v)  # existing atoms keep theirs
    ref = origami.Xoshiro256pp(7)
    mass = ch.topology().mass
    kbt = origami.BOLTZMANN_KJ_PER_MOL_K * 310.0
    expect = np.array([[math.sqrt(kbt * 1e-4 / mass[i]) * ref.gaussian() for _ in range(3)]
                       for i in range(ch.n_atoms)])
    np.testing.assert_array_equal(v2, expect)
