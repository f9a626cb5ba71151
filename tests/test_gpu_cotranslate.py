"""Co-translation on the GPU: the engine's exit-tunnel force (og_set_tunnel)
against the oracle restatement of CylindricalTunnel::add_force, and the
driver growing a chain (cotranslate.rs tests: cotranslate_ala3_grows_to_three_residues).

Tolerance: the tunnel force enters the 64-bit fixed-point accumulators
(2^-32 kJ/mol/A per unit), so force differences agree to 1e-8."""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))

import cotranslate as oracle_tunnel  # noqa: E402

pytestmark = pytest.mark.gpu


def forces_with(origami, chain, x, tunnel):
    eng = origami.Engine(origami.Params())
    eng.add_system(chain, x)
    eng.finalize()
    if tunnel is not None:
        tunnel.apply_to(eng)
    f = eng.total_force(0)
    eng.close()
    return f


def test_tunnel_force_matches_oracle(origami):
    from origami_b200.cotranslate import CylindricalTunnel
    ch = origami.Chain.build("NLYIQWLKDGGPSSGRPPPS")
    x = ch.positions - ch.positions.mean(axis=0)
    # a tilted axis along the extended chain, ending half-way along it: atoms
    # inside the radius, outside it, and beyond the tunnel's far end
    d = np.array([0.96, 0.28, 0.0]) / np.linalg.norm([0.96, 0.28, 0.0])
    tun = CylindricalTunnel(axis_origin=(-20.0, 0.0, 0.0), axis_direction=tuple(d), radius_a=4.0, length_a=35.0,
                            k_confine=25.0)
    ref = oracle_tunnel.tunnel_forces(x, tun.axis_origin, tun.axis_direction, tun.radius_a, tun.length_a,
                                      tun.k_confine)
    assert (np.abs(ref).sum(axis=1) > 0).sum() > 20 and (np.abs(ref).sum(axis=1) == 0).sum() > 20
    d = forces_with(origami, ch, x, tun) - forces_with(origami, ch, x, None)
    np.testing.assert_allclose(d, ref, atol=1e-8)


def test_tunnel_reference_cases(origami):
    """The reference's two tunnel tests, on one atom of a chain whose other
    atoms sit beyond the tunnel's axial extent."""
    from origami_b200.cotranslate import CylindricalTunnel
    ch = origami.Chain.build("A")
    x = ch.positions - ch.positions[1] + np.array([6.0, 0.0, 25.0])
    x[np.arange(ch.n_atoms) != 1, 2] += 200.0  # everything but CA out of [0, length]
    x[1] = [6.0, 0.0, 25.0]
    tun = CylindricalTunnel(radius_a=5.0, length_a=50.0, k_confine=10.0)
    d = forces_with(origami, ch, x, tun) - forces_with(origami, ch, x, None)
    np.testing.assert_allclose(d[1], [-10.0, 0.0, 0.0], atol=1e-8)
    assert np.abs(np.delete(d, 1, axis=0)).max() == 0.0
    x[1] = [2.0, 0.0, 40.0]
    d = forces_with(origami, ch, x, CylindricalTunnel()) - forces_with(origami, ch, x, None)
    assert np.abs(d).max() == 0.0


def test_cotranslate_ala3_grows_to_three_residues(origami):
    from origami_b200.cotranslate import UniformRibosome, run_cotranslate
    r = UniformRibosome("AAA", 50.0)
    opts = origami.LangevinOptions(dt_fs=1.0, temperature_k=310.0, friction_ps_inv=2.0, steps=0, save_every=10,
                                   seed=1, randomise_initial_velocities=True, include_sasa=False,
                                   constrain_h_bonds=False)
    frames = []
    final = run_cotranslate(r, opts, 50, None, lambda fr: frames.append(fr))
    assert final.n_residues == 3
    assert len(frames) > 5
    assert all(fr.residue_count <= 3 for fr in frames)
    assert np.isfinite(final.positions).all()
    times = [fr.time_fs for fr in frames]
    assert times == sorted(times) and times[-1] == pytest.approx(150.0)


def test_cotranslate_in_tunnel_stays_confined(origami):
    """A chain grown inside a narrow tunnel: after growth every atom still in
    the tunnel's axial extent is near the radius or inside it."""
    from origami_b200.cotranslate import CylindricalTunnel, UniformRibosome, run_cotranslate
    # origami's builder grows the chain along +x: the tunnel axis follows it
    tun = CylindricalTunnel(axis_origin=(-5.0, 0.0, 0.0), axis_direction=(1.0, 0.0, 0.0), radius_a=8.0,
                            length_a=60.0, k_confine=50.0)
    opts = origami.LangevinOptions(dt_fs=1.0, temperature_k=310.0, friction_ps_inv=2.0, save_every=50, seed=3)
    final = run_cotranslate(UniformRibosome("GSAGSAGS", 100.0), opts, 200, tun)
    x = final.positions - np.array(tun.axis_origin)
    along = x[:, 0]
    radial = np.linalg.norm(x[:, 1:], axis=1)
    inside = (along >= 0.0) & (along <= tun.length_a)
    assert np.isfinite(x).all()
    assert radial[inside].max() < tun.radius_a + 3.0
