#!/usr/bin/env python3
"""Regenerates tests/golden/known_answers.json from the reference's sources.

origami's own tests store no golden force or energy vectors, and the Rust
reference cannot be built here, so the checked numbers are the known answers
its tests, constants and README state.  This script reads each one where the
reference states it (file and line recorded beside the value) and writes the
JSON the oracle and host-model tests load.  Run it from the repository root
with the reference checkout's path:

    python tests/golden/make_known_answers.py /path/to/origami

The committed JSON is what the tests use; the script only needs the
reference when the fixture is refreshed.
"""
from __future__ import annotations

import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def find(root: str, rel: str, pattern: str, group: int = 1, flags: int = 0):
    """First match of `pattern` in reference file `rel`: (text, 'rel:line')."""
    with open(os.path.join(root, rel), encoding="utf-8") as f:
        text = f.read()
    m = re.search(pattern, text, flags)
    if not m:
        raise SystemExit(f"pattern not found in {rel}: {pattern}")
    line = text.count("\n", 0, m.start(group)) + 1
    return m.group(group), f"{rel}:{line}"


def num(s: str) -> float:
    return float(s.replace(",", "").replace("−", "-").replace("_f64", "").replace("_", ""))


def extract(root: str) -> dict:
    """Every known answer, read from the reference checkout at `root`."""
    out = {}

    def put(key, value, source, note):
        out[key] = {"value": value, "source": source, "note": note}

    v, src = find(root, "crates/energy/src/nonbonded.rs", r"assert_relative_eq!\(coul_kj,\s*(-?[\d.]+)")
    put("coulomb_unit_pair_5A_kj", num(v), src,
        "+1e / -1e at 5 A, no cutoff: -332.0637 / 5 * 4.184 kJ/mol (test tolerance 0.01)")
    v, src = find(root, "crates/dynamics/tests/trp_cage_minimise.rs", r"\+(\d+) kJ/mol structure")
    put("trp_cage_extended_total_kj", num(v), src, "extended Trp-cage total energy (no SASA)")
    v, src = find(root, "crates/dynamics/tests/trp_cage_minimise.rs", r"\+(\d+) kJ/mol to under")
    put("trp_cage_extended_bond_kj", num(v), src, "bond term of the extended Trp-cage")
    v, src = find(root, "README.md", r"drops the energy from \+([\d,]+) kJ/mol")
    put("readme_extended_total_kj", num(v), src, "the README's figure for the same structure")
    v, src = find(root, "README.md", r"to\s*\n?\s*([−-][\d,]+) kJ/mol in \d+ steps")
    put("readme_lbfgs_final_kj", num(v), src, "L-BFGS on the extended Trp-cage (history sensitive)")
    v, src = find(root, "README.md", r"kJ/mol in (\d+) steps")
    put("readme_lbfgs_steps", int(v), src, "L-BFGS steps to that energy")
    v, src = find(root, "crates/dynamics/tests/trp_cage_minimise.rs", r"result\.final_energy < ([\d.]+)")
    put("trp_cage_minimised_total_below_kj", num(v), src, "acceptance bound after L-BFGS (max 500 steps, gtol 5)")
    v, src = find(root, "crates/dynamics/tests/trp_cage_minimise.rs", r"result\.steps < (\d+)")
    put("trp_cage_minimise_steps_below", int(v), src, "acceptance bound on L-BFGS steps")
    v, src = find(root, "crates/dynamics/tests/trp_cage_minimise.rs", r"bond_kj_mol < ([\d.]+)")
    put("trp_cage_minimised_bond_below_kj", num(v), src, "bond term bound after L-BFGS")
    for key, const in (("n_ca_a", "N_CA"), ("ca_c_a", "CA_C"), ("c_o_a", "C_O"), ("peptide_c_n_a", "PEPTIDE_C_N")):
        v, src = find(root, "crates/geom/src/builder.rs", rf"const {const}: f64 = ([\d.]+);")
        put(f"backbone_{key}", num(v), src, f"builder bond length {const}")
    v, src = find(root, "crates/energy/src/sasa.rs", r"pub const PROBE_RADIUS_A: f64 = ([\d.]+);")
    put("sasa_probe_radius_a", num(v), src, "solvent probe radius")
    v, src = find(root, "crates/energy/src/sasa.rs", r"fn isolated_carbon_full_sphere[\s\S]*?\(([\d.]+)_f64 \+ [\d.]+\)\.powi\(2\)")
    put("sasa_isolated_carbon_vdw_a", num(v), src, "isolated carbon: area 4 pi (vdW + probe)^2")
    v, src = find(root, "crates/dynamics/tests/cotranslate_acceptance.rs", r"assert_eq!\(final_s\.atom_count\(\), (\d+)\)")
    put("cotranslate_agaga_atoms", int(v), src, "Ala-Gly-Ala-Gly-Ala grown by cotranslate")
    v, src = find(root, "README.md", r"native 1L2Y an energy ([\d,]+) kJ/mol below")
    put("readme_native_1l2y_gap_kj", num(v), src, "extended minus native 1L2Y total (no SASA)")
    for key, name, pat in (
            ("m7_chignolin_min_gap_kj", "GYDPETGTWG", r"\"GYDPETGTWG\",\s*([\d.]+),"),
            ("m7_trp_cage_min_gap_kj", "NLYIQWLKDGGPSSGRPPPS", r"\"NLYIQWLKDGGPSSGRPPPS\",\s*([\d.]+),"),
            ("m7_villin_min_gap_kj", "villin", r"gap > ([\d_.]+),\s*\n\s*\"villin")):
        v, src = find(root, "crates/io/tests/m7_native_vs_extended.rs", pat)
        put(key, num(v), src, f"native {name} scores at least this far below the extended build")
    v, src = find(root, "crates/io/tests/m7_native_vs_extended.rs", r"max_steps: (\d+),\s*\n\s*gradient_tol: ([\d.]+)")
    put("m7_villin_lbfgs_steps", int(v), src, "L-BFGS steps on the villin fixture before scoring (gtol 50, "
        "energy tol 1, max step 0.1 A)")
    v, src = find(root, "crates/energy/src/nonbonded.rs", r"pub const DEFAULT_CUTOFF_A: f64 = ([\d.]+);")
    put("nonbonded_default_cutoff_a", num(v), src, "LJ / Coulomb cutoff of the energy the pins use")
    return out


def main(root: str) -> None:
    out = extract(root)
    path = os.path.join(HERE, "known_answers.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
        f.write("\n")
    print(f"wrote {len(out)} known answers to {path}")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit(__doc__)
    main(sys.argv[1])
