#!/usr/bin/env python3
"""Writes tests/golden/bench_chain_300.npz: the benchmark's system, so that
the GPU arm and the CPU arms of bench.py time exactly the same input.

The system is the seeded-uniform 300-residue chain (xoshiro256++ seed 0 over
AminoAcid::ALL, 4 694 atoms with hydrogens), built extended by NeRF and
relaxed: L-BFGS on the GPU engine (all pairs, at most 300 steps, gradient
L-inf < 5 kJ/mol/A) and then 200 steps of overdamped Langevin at 100 K
(dt 0.5 fs, friction 50 ps^-1), as origami minimises before dynamics.  The
file holds the sequence, the relaxed coordinates and every og_topology array
of the chain (keys "topo_<field>", the layout of tests/golden/host_model.npz).

Needs a CUDA device and the built library:

    python tests/golden/make_bench_chain.py [OUT.npz]
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

FIELDS = ("charge", "rmin_half", "epsilon", "rmin_half_14", "epsilon_14", "gb_rho", "gb_scale", "mass", "element",
          "bonds", "bond_k", "bond_r0", "angles", "angle_k", "angle_theta0", "dihedrals", "dihedral_term_start",
          "term_k", "term_n", "term_delta", "impropers", "improper_k", "improper_psi0", "exclusions",
          "exclusion_kind", "constraints", "constraint_length")


def main(out: str) -> None:
    import bench
    import origami_b200 as og
    seq = bench.seeded_sequence(300, 0)
    chain = og.Chain.build(seq)
    res = bench.relax(og, chain, all_pairs=True)
    t = chain.topology()
    arrays = {"topo_" + f: np.asarray(getattr(t, f)) for f in FIELDS}
    np.savez_compressed(out, seq=np.array(seq), xyz=chain.positions, **arrays)
    print(f"wrote {out}: {chain.n_atoms} atoms, L-BFGS {res.initial_energy:.1f} -> {res.final_energy:.1f} kJ/mol "
          f"in {res.steps} steps")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "bench_chain_300.npz"))
