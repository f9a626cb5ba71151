"""Host model (sequence -> chain -> topology -> per-atom parameters) against
origami's own tests and known answers.  CPU only."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
import pytest

from conftest import ROOT, oracle, known

# a reference checkout, when one is named (the regeneration check needs it)
REF = os.environ.get("ORIGAMI_REFERENCE_DIR", "")


def names_of(chain):
    return [chain.atom_info(i)[2] for i in range(chain.n_atoms)]


def index_of(chain, residue, name):
    for i in range(chain.n_atoms):
        r, _, n = chain.atom_info(i)
        if r == residue and n == name:
            return i
    raise KeyError((residue, name))


def bondset(topo):
    return {tuple(b) for b in topo.bonds.tolist()}


def test_all_twenty_residue_atom_count(origami):
    # 324 atoms for one of each of the 20 amino acids (io/tests/build_all_residues.rs)
    ch = origami.Chain.build("ARNDCQEGHILKMFPSTWYV")
    assert ch.n_residues == 20
    assert ch.n_atoms == 324
    assert ch.missing_params() == 0


def test_agaga_has_44_atoms(origami):
    # dynamics/tests/cotranslate_acceptance.rs:47-49
    assert origami.Chain.build("AGAGA").n_atoms == known("cotranslate_agaga_atoms") == 44


def test_backbone_bond_lengths(origami):
    # io/tests/build_all_residues.rs:22-37: NeRF backbone lengths exact to 1e-6
    ch = origami.Chain.build("ARNDCQEGHILKMFPSTWYV")
    x = ch.positions
    for r in range(20):
        n, ca, c, o = (index_of(ch, r, a) for a in ("N", "CA", "C", "O"))
        assert abs(np.linalg.norm(x[ca] - x[n]) - known("backbone_n_ca_a")) < 1e-6
        assert abs(np.linalg.norm(x[c] - x[ca]) - known("backbone_ca_c_a")) < 1e-6
        assert abs(np.linalg.norm(x[o] - x[c]) - known("backbone_c_o_a")) < 1e-6
        if r > 0:
            pc = index_of(ch, r - 1, "C")
            assert abs(np.linalg.norm(x[n] - x[pc]) - known("backbone_peptide_c_n_a")) < 1e-6


def test_no_clashes_in_extended_chain(origami):
    # io/tests/build_all_residues.rs:40-55: no two atoms closer than 0.7 A
    x = origami.Chain.build("ARNDCQEGHILKMFPSTWYV").positions
    d = np.linalg.norm(x[:, None] - x[None], axis=-1) + np.eye(len(x)) * 10
    assert d.min() > 0.7


def test_alanine_and_glycine_bond_counts(origami):
    # geom/src/topology_graph.rs tests alanine_bond_count / glycine_bond_count
    assert len(origami.Chain.build("A").topology().bonds) == 9
    assert len(origami.Chain.build("G").topology().bonds) == 6


def test_ring_closures_and_peptide_bond(origami):
    ch = origami.Chain.build("AP")
    b = bondset(ch.topology())
    n, cd = index_of(ch, 1, "N"), index_of(ch, 1, "CD")
    assert (min(n, cd), max(n, cd)) in b
    c0, n1 = index_of(ch, 0, "C"), index_of(ch, 1, "N")
    assert (c0, n1) in b
    phe = origami.Chain.build("F")
    b = bondset(phe.topology())
    ring = ["CG", "CD1", "CE1", "CZ", "CE2", "CD2"]
    for a1, a2 in zip(ring, ring[1:] + ring[:1]):
        i, j = index_of(phe, 0, a1), index_of(phe, 0, a2)
        assert (min(i, j), max(i, j)) in b


def test_exclusions_match_graph_predicates(origami):
    # ForceScratch::rebuild_exclusions (scratch.rs:233) classifies every pair with
    # the TopologyGraph predicates; the host's list must be identical (bit-exact).
    for seq in ("AKE", "PWHFY", "NLYIQWLKDGGPSSGRPPPS", "CC"):
        ch = origami.Chain.build(seq)
        t = ch.topology()
        n = t.n_atoms
        ref = np.zeros((n, n), dtype=np.int8)
        bonds = np.ascontiguousarray(t.bonds.astype(np.int32))
        oracle().orc_exclusion_matrix(n, len(bonds), bonds.ctypes.data_as(C.POINTER(C.c_int32)),
                                      ref.ctypes.data_as(C.POINTER(C.c_int8)))
        got = np.zeros((n, n), dtype=np.int8)
        got[t.exclusions[:, 0], t.exclusions[:, 1]] = t.exclusion_kind
        got[t.exclusions[:, 1], t.exclusions[:, 0]] = t.exclusion_kind
        assert np.array_equal(got, ref), seq
        assert np.all(t.exclusions[:, 0] < t.exclusions[:, 1])


def test_one_three_and_one_four(origami):
    # geom/src/topology_graph.rs test one_three_and_one_four_exclusions
    ch = origami.Chain.build("A")
    t = ch.topology()
    kind = {(int(i), int(j)): int(k) for (i, j), k in zip(t.exclusions, t.exclusion_kind)}
    n, ca, c, o = (index_of(ch, 0, a) for a in ("N", "CA", "C", "O"))
    assert kind[(min(n, ca), max(n, ca))] == 1
    assert kind[(min(n, c), max(n, c))] == 1      # 1-3
    assert kind[(min(n, o), max(n, o))] == 2      # 1-4


def test_disulfide_detection(origami):
    ch = origami.Chain.build("CC")
    sg0, sg1 = index_of(ch, 0, "SG"), index_of(ch, 1, "SG")
    assert (sg0, sg1) not in bondset(ch.topology())
    x = ch.positions
    x[sg1] = x[sg0] + np.array([2.0, 0.0, 0.0])
    ch.positions = x
    # topology is rebuilt from positions when the chain changes
    ch.append("A")
    assert (sg0, sg1) in bondset(ch.topology())


def test_improper_lists(origami):
    # peptide C (one per peptide bond) + Asn CG, Gln CD, Asp CG, Glu CD, Arg CZ
    t = origami.Chain.build("NQDER").topology()
    assert len(t.impropers) == 4 + 5


def test_parameters_known_values(origami):
    # chem/src/forcefield.rs tests: C nonbonded eps 0.11 Rmin/2 2.0; Ala N -0.47, CA 0.07, H 0.31
    ch = origami.Chain.build("A")
    t = ch.topology()
    i = {ch.atom_info(k)[2]: k for k in range(ch.n_atoms)}
    assert abs(t.charge[i["N"]] + 0.47) < 1e-12
    assert abs(t.charge[i["CA"]] - 0.07) < 1e-12
    assert abs(t.charge[i["H"]] - 0.31) < 1e-12
    assert abs(t.epsilon[i["C"]] - 0.11) < 1e-12 and abs(t.rmin_half[i["C"]] - 2.0) < 1e-12
    # X-H constraints: every H bonded once, target = force-field r0
    assert len(t.constraints) == sum(1 for k in range(ch.n_atoms) if t.element[k] == 0)
    # GB intrinsic radii / HCT scales (gb.rs:58-83)
    assert abs(t.gb_rho[i["O"]] - 1.50) < 1e-12 and abs(t.gb_scale[i["O"]] - 0.85) < 1e-12


def test_histidine_is_hsd(origami):
    ch = origami.Chain.build("H")
    t = ch.topology()
    i = {ch.atom_info(k)[2]: k for k in range(ch.n_atoms)}
    assert "HD1" in i and "HE2" not in i
    assert abs(t.charge[i["HD1"]] - 0.32) < 0.02


@pytest.mark.skipif(not REF or not os.path.isdir(REF), reason="no reference checkout named")
def test_tables_regenerate_identically(tmp_path):
    """The committed tables are exactly what make_tables.py derives from the reference."""
    import importlib.util
    import shutil
    spec = importlib.util.spec_from_file_location("mt", os.path.join(ROOT, "origami_b200", "data", "make_tables.py"))
    mt = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mt)
    with open(os.path.join(REF, "crates/chem/src/topology_data.rs")) as fh:
        tpl = mt.parse_templates(fh.read())
    out = tmp_path / "t.tbl"
    mt.write_templates(tpl, str(out))
    assert out.read_text() == open(os.path.join(ROOT, "origami_b200", "data", "residue_templates.tbl")).read()
    with open(os.path.join(REF, "data/charmm36/par_all36m_prot.prm")) as fh:
        recs = mt.parse_prm(fh.read())
    committed = open(os.path.join(ROOT, "origami_b200", "data", "charmm36m_protein.ff")).read().splitlines()
    assert [l for l in committed if not l.startswith(("#", "CHARGE"))] == recs
    del shutil
