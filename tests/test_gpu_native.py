"""The GPU on the reference's native structures: the PDB fixtures read by the
independent oracle (tests/golden/host_model.npz: chignolin 1UAO, Trp-cage
1L2Y, villin 2F4K, crambin 1CRN with three disulfides, insulin 2HIU with two
chains), built by the product through og_chain_from_structure, against the
FP64 oracle running on the oracle's own topology arrays.  These are compact
folds, unlike the extended or relaxed NeRF builds the other parity tests
use.  Tolerances as elsewhere: forces RMS relative < 1e-5, energies per term
< 1e-6 relative, surface areas < 1e-9 of 4 pi R^2.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import INF, GoldenSystem, Orc, dp, host_golden, oracle

pytestmark = pytest.mark.gpu

FIXTURES = ("1UAO", "1L2Y", "2F4K", "1CRN", "2HIU")
TERMS = ("bond", "angle", "dihedral", "improper", "lj", "coulomb", "gb", "gb_self", "gb_pair", "total")


def rms_rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


def _chain(origami, case):
    return origami.Chain.from_structure(str(case["seq"]), case["counts"], [str(n) for n in case["names"]],
                                        case["xyz"], elements=case["elements"], chains=str(case["chains"]))


@pytest.mark.parametrize("name", FIXTURES)
@pytest.mark.parametrize("mode", ["all_pairs", "cutoff"])
def test_native_forces_and_energies_match_oracle(origami, name, mode):
    case = host_golden()[name]
    ch = _chain(origami, case)
    x = np.asarray(case["xyz"], dtype=np.float64)
    params = origami.Params.all_pairs() if mode == "all_pairs" else origami.Params()
    eng = origami.Engine(params)
    eng.add_system(ch, x)
    eng.finalize()
    f = eng.total_force(0)
    e = eng.energies(0)
    eng.close()
    orc = Orc(GoldenSystem(case))
    cut = (INF, INF, INF) if mode == "all_pairs" else (10.0, 20.0, 10.0)
    assert rms_rel(f, orc.total_force(x, *cut)) < 1e-5
    ref = orc.energy_terms(x, cut[0], cut[1])
    for k in TERMS:
        assert abs(e[k] - ref[k]) / max(abs(ref[k]), 1.0) < 1e-6, (name, k, e[k], ref[k])


@pytest.mark.parametrize("name", ("1L2Y", "2HIU"))
def test_native_surface_areas_match_oracle(origami, name):
    case = host_golden()[name]
    ch = _chain(origami, case)
    x = np.ascontiguousarray(case["xyz"], dtype=np.float64)
    eng = origami.Engine(origami.Params())
    eng.add_system(ch, x)
    eng.finalize()
    got = eng.sasa_areas(0, "powersasa")
    eng.close()
    o = oracle()
    rad = np.array([o.orc_sasa_radius(int(el)) for el in case["elements"]])
    ref = np.zeros(ch.n_atoms)
    o.orc_sasa_areas(ch.n_atoms, dp(x), dp(rad), dp(ref))
    assert np.max(np.abs(got - ref) / (4 * np.pi * rad ** 2)) < 1e-9
