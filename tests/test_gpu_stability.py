"""Long MD with the surface term: the bench's seeded 300-residue chain,
L-BFGS-relaxed, 16 replicas at 310 K, dt 2 fs + SHAKE, PowerSasa on, for 500
steps in all-pairs and in cutoff mode.  Every replica must stay finite and
SHAKE must converge every step.  CH2 groups under SHAKE pass through the
tangent band of the surface term (two H caps touching on the C sphere)
regularly; with the reference's proximity rule for those vertices one
replica of the cutoff-mode bench diverged within 100 steps."""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


@pytest.mark.parametrize("cutoff", [False, True])
def test_sasa_md_stays_finite_and_shake_converges(origami, cutoff):
    import bench
    seq, chain = bench.build_workload(origami, 300, 0)
    bench.relax(origami, chain, all_pairs=not cutoff)
    mk = origami.Params if cutoff else origami.Params.all_pairs
    p = mk(dt_fs=2.0, friction_ps_inv=2.0, constrain_h_bonds=True, seed=11, include_sasa=True,
           sasa_gamma_scale=0.25)
    eng = origami.Engine(p)
    for _ in range(16):
        eng.add_system(chain, chain.positions, 310.0)
    eng.finalize()
    for r in range(16):
        eng.init_velocities(r, 1000 + r, remove_com=False)
    eng.step(500)
    for r in range(16):
        s = eng.stats(r)
        assert not s["diverged"] and s["shake_failures"] == 0, (r, s)
        assert np.isfinite(eng.positions(r)).all() and np.isfinite(eng.velocities(r)).all()
        assert 150.0 < eng.kinetic(r)[1] < 450.0
    eng.close()
