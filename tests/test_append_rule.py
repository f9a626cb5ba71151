"""The rule an engine system grows by (og_topology_extends, host only): the
topology of a chain after og_chain_append (cotranslate.rs:204, the residue
the ribosome emits) extends the topology before it -- the old atoms keep
their parameters and every term among them stays, in order -- and topologies
that change an old atom or drop an old term do not.
"""
from __future__ import annotations

import dataclasses

import numpy as np

import origami_b200 as og


def _copy(t: og.Topology) -> og.Topology:
    return dataclasses.replace(t, **{f.name: getattr(t, f.name).copy() for f in dataclasses.fields(t)
                                     if f.name != "_keep"}, _keep=[])


def test_each_append_extends_the_previous_topology():
    ch = og.Chain.build("M")
    prev = ch.topology()
    for aa in "ACDEFGHIKLMNPQRSTVWY":  # every residue type once
        ch.append(aa)
        cur = ch.topology()
        ok, why = og.topology_extends(prev, cur)
        assert ok, (aa, why)
        # the new records are exactly those touching a new atom
        n_old = prev.n_atoms
        for arr, old in ((cur.bonds, prev.bonds), (cur.angles, prev.angles), (cur.dihedrals, prev.dihedrals),
                         (cur.impropers, prev.impropers), (cur.exclusions, prev.exclusions),
                         (cur.constraints, prev.constraints)):
            old_only = arr[(arr < n_old).all(axis=1)] if len(arr) else arr
            assert np.array_equal(old_only, old)
        prev = cur


def test_chain_objects_are_accepted_directly():
    a = og.Chain.build("GAV")
    b = og.Chain.build("GAV")
    b.append("L")
    assert og.topology_extends(a, b) == (True, "")
    assert og.topology_extends(b, a)[0] is False  # fewer atoms


def test_changes_to_old_atoms_or_terms_are_refused():
    ch = og.Chain.build("GAVL")
    base = ch.topology()
    ch.append("K")
    grown = ch.topology()

    t = _copy(grown)
    t.charge[3] += 1e-9
    ok, why = og.topology_extends(base, t)
    assert not ok and "parameters" in why

    t = _copy(grown)
    keep = ~((t.bonds[:, 0] == base.bonds[0, 0]) & (t.bonds[:, 1] == base.bonds[0, 1]))
    t.bonds, t.bond_k, t.bond_r0 = t.bonds[keep], t.bond_k[keep], t.bond_r0[keep]
    ok, why = og.topology_extends(base, t)
    assert not ok and "bonds" in why

    t = _copy(grown)
    old = np.flatnonzero((t.angles < base.n_atoms).all(axis=1))
    t.angle_k[old[5]] *= 1.5
    ok, why = og.topology_extends(base, t)
    assert not ok and "angles" in why

    t = _copy(grown)
    old = np.flatnonzero((t.exclusions < base.n_atoms).all(axis=1))
    t.exclusion_kind[old[0]] = 3 - t.exclusion_kind[old[0]]
    ok, why = og.topology_extends(base, t)
    assert not ok and "exclusions" in why

    t = _copy(grown)
    old = np.flatnonzero((t.dihedrals < base.n_atoms).all(axis=1))
    t.term_k[t.dihedral_term_start[old[2]]] += 0.25  # one Fourier term of an old dihedral
    ok, why = og.topology_extends(base, t)
    assert not ok and "dihedrals" in why

    t = _copy(grown)
    old = np.flatnonzero((t.constraints < base.n_atoms).all(axis=1))
    t.constraint_length[old[1]] *= 1.01
    ok, why = og.topology_extends(base, t)
    assert not ok and "constraints" in why

    t = _copy(grown)  # an old improper dropped
    old = np.flatnonzero((t.impropers < base.n_atoms).all(axis=1))
    keep = np.ones(len(t.improper_k), bool)
    keep[old[0]] = False
    t.impropers, t.improper_k, t.improper_psi0 = t.impropers[keep], t.improper_k[keep], t.improper_psi0[keep]
    ok, why = og.topology_extends(base, t)
    assert not ok and "impropers" in why

    ok, why = og.topology_extends(base, base)
    assert not ok and "no new atoms" in why
