"""The co-translation workload at full scale: a chain of 10 000+ atoms (the
first 640 residues of the seeded sequence the 1000-residue run grows) with
the surface term (gamma scale 0.25) and the exit tunnel, all pairs.  Forces
against the FP64 oracle (pair terms, PowerSasa, tunnel: RMS relative < 1e-5),
then the cotranslation driver appends residues to it and steps on.
"""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

from conftest import INF, Orc, dp, oracle

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))

import cotranslate as oracle_tunnel  # noqa: E402

pytestmark = pytest.mark.gpu


def rms_rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


def _sequence(n):
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    return bench.seeded_sequence(n, 0)


def test_forces_of_a_10k_atom_chain_with_surface_term_and_tunnel(origami):
    from origami_b200.cotranslate import CylindricalTunnel
    ch = origami.Chain.build(_sequence(640))
    assert ch.n_atoms >= 10_000
    x = ch.positions + np.random.default_rng(64).normal(scale=0.02, size=(ch.n_atoms, 3))
    tun = CylindricalTunnel(axis_origin=(-5.0, 0.0, 0.0), axis_direction=(1.0, 0.0, 0.0), radius_a=10.0,
                            length_a=80.0, k_confine=10.0)
    eng = origami.Engine(origami.Params.all_pairs(include_sasa=True, sasa_gamma_scale=0.25))
    eng.add_system(ch, x)
    eng.finalize()
    tun.apply_to(eng)
    f_gpu = eng.total_force(0)
    eng.close()
    orc = Orc(ch)
    f_ref = orc.total_force(x, INF, INF, INF)
    el = ch.topology().element
    o = oracle()
    rad = np.array([o.orc_sasa_radius(int(e)) for e in el])
    gam = np.array([o.orc_sasa_gamma(int(e), 0.25) for e in el])
    fs = np.zeros_like(x)
    o.orc_sasa_forces_tangent_one_root(x.shape[0], dp(np.ascontiguousarray(x)), dp(rad), dp(gam), dp(fs))
    ft = oracle_tunnel.tunnel_forces(x, tun.axis_origin, tun.axis_direction, tun.radius_a, tun.length_a,
                                     tun.k_confine)
    assert (np.abs(ft).sum(axis=1) > 0).any()
    err = rms_rel(f_gpu, f_ref + fs + ft)
    assert err < 1e-5, err


def test_cotranslation_continues_at_10k_atoms(origami):
    """Two more residues emitted onto a 10 000-atom chain by the driver's
    own steps (append, L-BFGS, new-atom velocities, a dynamics slice with
    SHAKE and the surface term): the chain grows and stays finite."""
    from origami_b200.cotranslate import CotranslateTimings, _run_slice
    from origami_b200.minimize import minimize_chain
    from origami_b200.cotranslate import APPEND_MINIMIZE, seed_new_atom_velocities
    seq = _sequence(642)
    ch = origami.Chain.build(seq[:640])
    base = origami.Params.all_pairs(sasa_gamma_scale=0.25)
    minimize_chain(ch, params=base, opts=APPEND_MINIMIZE)
    opts = origami.LangevinOptions(dt_fs=2.0, temperature_k=310.0, friction_ps_inv=2.0, save_every=0, seed=4,
                                   include_sasa=True, constrain_h_bonds=True)
    rng = origami.Xoshiro256pp(4)
    v = seed_new_atom_velocities(ch, np.zeros((0, 3)), 310.0, rng)
    t = CotranslateTimings()
    clock, done = 0.0, 0
    for aa in seq[640:]:
        ch.append(aa)
        minimize_chain(ch, params=base, opts=APPEND_MINIMIZE)
        v = seed_new_atom_velocities(ch, v, 310.0, rng)
        clock, done, v = _run_slice(ch, v, opts, 50, None, base, clock, done, ch.n_residues, None, timings=t)
    assert ch.n_residues == 642 and ch.n_atoms > 10_000
    assert np.isfinite(ch.positions).all() and np.isfinite(v).all()
    assert t.steps == 100 and t.slices == 2
