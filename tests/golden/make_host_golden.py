#!/usr/bin/env python3
"""Regenerates tests/golden/host_model.npz: origami's host model evaluated by
the independent oracle (oracle/host_model.py) straight from a reference
checkout -- its Rust tables and CHARMM36m files -- for fixed structures:

  ext_all20    the 20 residues in AminoAcid::ALL order, as the builder lays
               them out (atom names and elements only; an extended build has
               no disulfide, so its coordinates do not enter the topology)
  ext_1UAO ext_1L2Y ext_2F4K
               extended builds of those fixtures' sequences, likewise
  1UAO 1L2Y 2F4K 1CRN 2HIU
               the reference's PDB fixtures (crates/io/tests/fixtures/), read
               by the oracle's restatement of read_pdb: chignolin, Trp-cage
               model 1, villin HP35, crambin (three disulfides), insulin (two
               chains, TER between them)

For each: the structure (one-letter codes, chain ids, atoms per residue,
names, element codes, coordinates) and every og_topology array.  The CPU
tests rebuild each structure with the product and compare the arrays bit for
bit, and score the native fixtures with the FP64 oracle on these arrays.

    python tests/golden/make_host_golden.py /path/to/origami
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import host_model as hm  # noqa: E402

FIXTURES = {"1UAO": "1UAO_chignolin.pdb", "1L2Y": "1L2Y_model1.pdb", "2F4K": "2F4K_villin_hp35.pdb",
            "1CRN": "1CRN_crambin.pdb", "2HIU": "2HIU_insulin.pdb"}
EXTENDED = {"ext_all20": "ARNDCQEGHILKMFPSTWYV"}
EXTENDED_OF = ("1UAO", "1L2Y", "2F4K")  # fixtures with at most one Cys


def extended_structure(model: hm.HostModel, seq: str) -> list:
    assert seq.count("C") <= 1, "an extended build with two Cys would need its coordinates"
    nan = (float("nan"),) * 3
    return [(model.aa_variants[hm.AA_ONE.index(c)], "A",
             [(n, e, nan) for n, e in model.residue_atoms(model.aa_variants[hm.AA_ONE.index(c)])]) for c in seq]


def pack(model: hm.HostModel, residues: list) -> dict:
    topo = model.topology(residues)
    topo.pop("atom_type")
    out = {f"topo_{k}": v for k, v in topo.items()}
    out["seq"] = np.array("".join(hm.AA_ONE[model.aa_variants.index(aa)] for aa, _, _ in residues))
    out["chains"] = np.array("".join(ch for _, ch, _ in residues))
    out["counts"] = np.array([len(a) for _, _, a in residues], dtype=np.int32)
    out["names"] = np.array([n for _, _, a in residues for n, _, _ in a])
    out["elements"] = np.array([hm.ELEMENTS.index(e) for _, _, a in residues for _, e, _ in a], dtype=np.int32)
    out["xyz"] = np.array([p for _, _, a in residues for _, _, p in a], dtype=np.float64)
    return out


def generate(ref: str) -> dict:
    model = hm.HostModel(ref)
    cases = {}
    for key, seq in EXTENDED.items():
        cases[key] = pack(model, extended_structure(model, seq))
    for key, fname in FIXTURES.items():
        with open(os.path.join(ref, "crates/io/tests/fixtures", fname)) as fh:
            cases[key] = pack(model, hm.read_pdb(fh.read(), model))
    for key in EXTENDED_OF:
        cases["ext_" + key] = pack(model, extended_structure(model, str(cases[key]["seq"])))
    return {f"{c}/{k}": v for c, d in cases.items() for k, v in d.items()}


def main(ref: str) -> None:
    flat = generate(ref)
    path = os.path.join(HERE, "host_model.npz")
    np.savez_compressed(path, **flat)
    print(f"wrote {len(flat)} arrays to {path} ({os.path.getsize(path) / 1024:.0f} KiB)")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit(__doc__)
    main(sys.argv[1])
