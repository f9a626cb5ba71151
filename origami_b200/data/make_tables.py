#!/usr/bin/env python3
"""Generate the two data tables the host model loads at run time.

The GPU box that runs the engine has no copy of the origami source tree, so the
chemistry the engine needs travels with this package as two small text tables
written by this script:

* ``charmm36m_protein.ff`` -- every CHARMM36m parameter record that origami's
  parser accepts for the atom types it models, plus the per-(residue, atom)
  partial charges after origami's CHARMM->PDB atom-name translation.
* ``residue_templates.tbl`` -- the side-chain internal-coordinate templates of
  the 20 amino acids (NeRF parents, bond length, bond angle, dihedral rule) and
  each residue's default chi angles.

Both tables have to be *alike* the reference's: they are the chemistry. This
script restates the reference's parser rules (crates/chem/src/forcefield.rs:218-459,
``parse``/``parse_*_line``/``parse_rtf_charges``/``charmm_to_pdb_atom_name``) and
evaluates the const-fn template expressions of crates/chem/src/topology_data.rs
(helpers ``cb_atom`` :44, ``methyl_h`` :1509, ``beta_h`` :1532, ``ch2_chi`` :1554).
Only accepted parameter records are written, in file order, with their numeric
tokens unchanged, so the C++ loader (origami_b200/csrc/host/forcefield.cpp)
applies the reference's first-wins / append semantics to exactly the same
inputs.

Usage:  python origami_b200/data/make_tables.py REFERENCE_ROOT
(or with ORIGAMI_REFERENCE_DIR set).  Run it only where the reference source
is present; the outputs are committed.
"""
from __future__ import annotations

import math
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))

# AtomType enum of crates/chem/src/atom_type.rs:18-107 (declaration order = Ord).
ATOM_TYPES = [
    "C", "CA", "CAI", "CC", "CT1", "CT2", "CT2A", "CT3", "CP1", "CP2", "CP3",
    "CPH1", "CPH2", "CPT", "CY",
    "N", "NH1", "NH2", "NH3", "NC2", "NR1", "NR2", "NY",
    "O", "OC", "OH1",
    "S",
    "H", "HA", "HA1", "HA2", "HA3", "HB1", "HB2", "HC", "HP", "HR1", "HR3", "HS",
]
TYPE_SET = set(ATOM_TYPES)

# AminoAcid::ALL order (crates/chem/src/amino_acid.rs:31).
AA3 = ["ALA", "ARG", "ASN", "ASP", "CYS", "GLN", "GLU", "GLY", "HIS", "ILE",
       "LEU", "LYS", "MET", "PHE", "PRO", "SER", "THR", "TRP", "TYR", "VAL"]
RTF_RESI = {"ALA": "ALA", "ARG": "ARG", "ASN": "ASN", "ASP": "ASP", "CYS": "CYS",
            "GLN": "GLN", "GLU": "GLU", "GLY": "GLY", "HSD": "HIS", "ILE": "ILE",
            "LEU": "LEU", "LYS": "LYS", "MET": "MET", "PHE": "PHE", "PRO": "PRO",
            "SER": "SER", "THR": "THR", "TRP": "TRP", "TYR": "TYR", "VAL": "VAL"}


# ---------------------------------------------------------------------------
# Residue templates
# ---------------------------------------------------------------------------

def _split_top(s: str) -> list[str]:
    """Split on commas that sit outside (), {} and []."""
    out, depth, cur = [], 0, []
    for ch in s:
        if ch in "({[":
            depth += 1
        elif ch in ")}]":
            depth -= 1
        if ch == "," and depth == 0:
            out.append("".join(cur))
            cur = []
        else:
            cur.append(ch)
    if "".join(cur).strip():
        out.append("".join(cur))
    return [x.strip() for x in out if x.strip()]


def _block_after(text: str, start: int, open_ch: str, close_ch: str) -> tuple[str, int]:
    i = text.index(open_ch, start)
    depth = 0
    for k in range(i, len(text)):
        if text[k] == open_ch:
            depth += 1
        elif text[k] == close_ch:
            depth -= 1
            if depth == 0:
                return text[i + 1:k], k + 1
    raise ValueError("unbalanced block")


def parse_templates(src: str) -> dict[str, dict]:
    src = re.sub(r"//[^\n]*", "", src)
    pi = math.pi

    def d(deg):
        return deg * pi / 180.0

    env = {
        "d": d,
        "TRANS": pi,
        "GAUCHE_PLUS": pi / 3.0,
        "GAUCHE_MINUS": -pi / 3.0,
        "CB_DIHEDRAL": d(-122.55),
        "CB_ANGLE": d(110.5),
        # crates/chem/src/topology.rs bond:: / angle:: constants
        "bond_C_C": 1.530, "bond_C_C_AROMATIC": 1.390, "bond_C_N": 1.470,
        "bond_C_N_AROMATIC": 1.340, "bond_C_O": 1.420, "bond_C_O_CARBOXYL": 1.250,
        "bond_C_S": 1.810, "bond_S_H": 1.340, "bond_O_H": 0.960, "bond_N_H": 1.010,
        "bond_C_H_SP3": 1.090, "bond_C_H_SP2": 1.080,
        "angle_TETRAHEDRAL": 109.471_220_634_490_69 * pi / 180.0,
        "angle_TRIGONAL": 120.0 * pi / 180.0,
        "angle_PEPTIDE_C_N_CA": 121.7 * pi / 180.0,
        "angle_N_CA_C": 111.2 * pi / 180.0,
        "angle_CA_C_O": 120.8 * pi / 180.0,
        "angle_CA_C_N": 116.2 * pi / 180.0,
        "Fixed": lambda x: ("F", 0, x),
        "Chi": lambda n: ("C", n, 0.0),
        "ChiPlus": lambda n, off: ("P", n, off),
    }

    def ev(expr: str):
        e = expr.strip()
        e = e.replace("DihedralValue::", "").replace("bond::", "bond_").replace("angle::", "angle_")
        e = e.replace("Element::", "")
        return eval(e, {"__builtins__": {}}, env)  # noqa: S307 - trusted literal table

    def h_atom(name, c, b, a, dih, length_key="bond_C_H_SP3"):
        return dict(name=name, element="H", bond_to=c, angle_at=b, dihedral_to=a,
                    length=env[length_key], angle=env["angle_TETRAHEDRAL"], dih=dih)

    def entry(item: str) -> dict:
        item = item.strip()
        if item.startswith("cb_atom"):
            return dict(name="CB", element="C", bond_to="CA", angle_at="N", dihedral_to="C",
                        length=env["bond_C_C"], angle=env["CB_ANGLE"],
                        dih=("F", 0, env["CB_DIHEDRAL"]))
        m = re.match(r"(methyl_h|beta_h|ch2_chi)\s*\((.*)\)\s*$", item, re.S)
        if m:
            args = _split_top(m.group(2))
            name, c, b, a = (x.strip().strip('"') for x in args[:4])
            if m.group(1) in ("methyl_h", "beta_h"):
                return h_atom(name, c, b, a, ("F", 0, ev(args[4])))
            chi_n = int(args[4])
            sign = int(args[5])
            off = d(120.0) if sign >= 0 else d(-120.0)
            return h_atom(name, c, b, a, ("P", chi_n, off))
        m = re.match(r"SidechainAtom\s*\{(.*)\}\s*$", item, re.S)
        if not m:
            raise ValueError(f"unrecognised template entry: {item[:60]}")
        fields = {}
        for f in _split_top(m.group(1)):
            k, v = f.split(":", 1)
            fields[k.strip()] = v.strip()
        return dict(
            name=fields["name"].strip('"'),
            element=fields["element"].replace("Element::", "").strip(),
            bond_to=fields["bond_to"].strip('"'),
            angle_at=fields["angle_at"].strip('"'),
            dihedral_to=fields["dihedral_to"].strip('"'),
            length=float(ev(fields["bond_length_a"])),
            angle=float(ev(fields["bond_angle_rad"])),
            dih=ev(fields["dihedral"]),
        )

    out = {}
    for m in re.finditer(r"const\s+([A-Z]{3})\s*:\s*ResidueTopology\s*=\s*ResidueTopology", src):
        body, _ = _block_after(src, m.end(), "{", "}")
        sc_start = body.index("sidechain:")
        sc_body, after = _block_after(body, sc_start, "[", "]")
        rest = body[after:]
        chi_m = re.search(r"default_chi_rad:\s*&\[(.*?)\]", rest, re.S)
        chi = [float(ev(x)) for x in _split_top(chi_m.group(1))] if chi_m.group(1).strip() else []
        amide = re.search(r"has_amide_h:\s*(true|false)", rest).group(1) == "true"
        gly = re.search(r"is_glycine:\s*(true|false)", rest).group(1) == "true"
        atoms = [entry(x) for x in _split_top(sc_body)]
        out[m.group(1)] = dict(atoms=atoms, chi=chi, amide=amide, gly=gly)
    return out


def write_templates(tpl: dict, path: str) -> None:
    lines = [
        "# origami residue templates (generated by make_tables.py; do not edit)",
        "# RES <AA3> <has_amide_h 0|1> <is_glycine 0|1> <n_chi> <chi_rad...>",
        "# ATOM <name> <element> <bond_to> <angle_at> <dihedral_to> <bond_length_A> <bond_angle_rad> <F|C|P> <chi_n> <value_rad>",
    ]
    for aa in AA3:
        t = tpl[aa]
        chis = " ".join(repr(x) for x in t["chi"])
        lines.append(f"RES {aa} {int(t['amide'])} {int(t['gly'])} {len(t['chi'])} {chis}".rstrip())
        for a in t["atoms"]:
            kind, n, val = a["dih"]
            lines.append(
                f"ATOM {a['name']} {a['element']} {a['bond_to']} {a['angle_at']} {a['dihedral_to']} "
                f"{a['length']!r} {a['angle']!r} {kind} {n} {float(val)!r}")
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")


# ---------------------------------------------------------------------------
# Force-field parameters
# ---------------------------------------------------------------------------

def _is_f64(tok: str) -> bool:
    try:
        float(tok)
    except ValueError:
        return False
    # Rust's f64 parser rejects some forms Python accepts (e.g. "nan" works in
    # both, "1_0" only in Python); the CHARMM file never has those forms.
    return "_" not in tok


def _is_u32(tok: str) -> bool:
    return tok.isdigit()


def _atom(tok: str) -> str:
    if tok in ("X", "x"):
        return "X"
    return tok if tok in TYPE_SET else "?"


def parse_prm(text: str) -> list[str]:
    """Return the accepted parameter records, in file order."""
    headers = {"BONDS": "B", "ANGLES": "A", "DIHEDRALS": "D", "IMPROPER": "I",
               "IMPROPERS": "I", "CMAP": "-", "NONBONDED": "N", "HBOND": "-", "END": "E"}
    section = None
    recs: list[str] = []
    for raw in text.splitlines():
        line = raw.split("!", 1)[0].strip()
        if not line:
            continue
        first = line.split()[0]
        if first in headers:
            section = headers[first]
            if section == "E":
                break
            continue
        if section is None or section == "-":
            continue
        tok = line.split()
        if section == "B":
            if len(tok) < 4:
                continue
            a, b = _atom(tok[0]), _atom(tok[1])
            if a in ("X", "?") or b in ("X", "?") or not (_is_f64(tok[2]) and _is_f64(tok[3])):
                continue
            recs.append(f"BOND {a} {b} {tok[2]} {tok[3]}")
        elif section == "A":
            if len(tok) < 5:
                continue
            a, b, c = (_atom(t) for t in tok[:3])
            if any(x in ("X", "?") for x in (a, b, c)) or not (_is_f64(tok[3]) and _is_f64(tok[4])):
                continue
            recs.append(f"ANGLE {a} {b} {c} {tok[3]} {tok[4]}")
        elif section == "D":
            if len(tok) < 7:
                continue
            a, b, c, d = (_atom(t) for t in tok[:4])
            if not (_is_f64(tok[4]) and _is_u32(tok[5]) and _is_f64(tok[6])):
                continue
            specific = all(x not in ("X", "?") for x in (a, b, c, d))
            wildcard = a == "X" and d == "X" and b not in ("X", "?") and c not in ("X", "?")
            if specific or wildcard:
                recs.append(f"DIHEDRAL {a} {b} {c} {d} {tok[4]} {tok[5]} {tok[6]}")
        elif section == "I":
            if len(tok) < 7:
                continue
            a, b, c, d = (_atom(t) for t in tok[:4])
            if not (_is_f64(tok[4]) and _is_f64(tok[6])):
                continue
            specific = all(x not in ("X", "?") for x in (a, b, c, d))
            wildcard = a not in ("X", "?") and b == "X" and c == "X" and d not in ("X", "?")
            if specific or wildcard:
                recs.append(f"IMPROPER {a} {b} {c} {d} {tok[4]} {tok[6]}")
        elif section == "N":
            if "cutnb" in line or "ctofnb" in line:
                continue
            if len(tok) < 4:
                continue
            t = _atom(tok[0])
            if t in ("X", "?") or not (_is_f64(tok[2]) and _is_f64(tok[3])):
                continue
            e14 = r14 = "-"
            if len(tok) >= 7 and _is_f64(tok[5]) and _is_f64(tok[6]):
                e14, r14 = tok[5], tok[6]
            recs.append(f"NONBONDED {t} {tok[2]} {tok[3]} {e14} {r14}")
    return recs


def charmm_to_pdb(aa: str, name: str, tpl: dict) -> str:
    """crates/chem/src/forcefield.rs charmm_to_pdb_atom_name (+ return_static_name)."""
    if name == "HN":
        return "H"
    ch2_b = {"LEU", "MET", "PRO", "SER", "CYS", "ASN", "GLN", "ASP", "GLU", "LYS",
             "ARG", "HIS", "PHE", "TYR", "TRP"}
    table = {
        ("GLY", "HA1"): "HA2", ("GLY", "HA2"): "HA3",
        ("ILE", "CD"): "CD1", ("ILE", "HD1"): "HD11", ("ILE", "HD2"): "HD12",
        ("ILE", "HD3"): "HD13", ("ILE", "HG11"): "HG12", ("ILE", "HG12"): "HG13",
        ("SER", "HG1"): "HG", ("CYS", "HG1"): "HG",
    }
    if (aa, name) in table:
        return table[(aa, name)]
    if aa in ch2_b and name == "HB1":
        return "HB2"
    if aa in ch2_b and name == "HB2":
        return "HB3"
    if aa in {"MET", "PRO", "GLN", "GLU", "LYS", "ARG"} and name in ("HG1", "HG2"):
        return {"HG1": "HG2", "HG2": "HG3"}[name]
    if aa in {"PRO", "LYS", "ARG"} and name in ("HD1", "HD2"):
        return {"HD1": "HD2", "HD2": "HD3"}[name]
    if aa == "LYS" and name in ("HE1", "HE2"):
        return {"HE1": "HE2", "HE2": "HE3"}[name]
    if name in ("N", "CA", "C", "O", "HA"):
        return name
    for a in tpl[aa]["atoms"]:
        if a["name"] == name:
            return name
    return ""


def parse_rtf(text: str, tpl: dict) -> dict[tuple[str, str], str]:
    current = None
    charges: dict[tuple[str, str], str] = {}
    for raw in text.splitlines():
        line = raw.split("!", 1)[0].strip()
        if not line:
            continue
        tok = line.split()
        head = tok[0]
        if head == "RESI":
            current = RTF_RESI.get(tok[1] if len(tok) > 1 else "")
            continue
        if head == "PRES":
            current = None
            continue
        if head != "ATOM" or current is None:
            continue
        name = tok[1] if len(tok) > 1 else ""
        q = tok[3] if len(tok) > 3 else ""
        if not _is_f64(q):
            continue
        pdb = charmm_to_pdb(current, name, tpl)
        charges[(current, pdb)] = q  # HashMap::insert: last write wins
    return charges


def main(argv: list[str]) -> int:
    ref = argv[1] if len(argv) > 1 else os.environ.get("ORIGAMI_REFERENCE_DIR", "")
    if not ref:
        raise SystemExit(__doc__)
    with open(os.path.join(ref, "crates/chem/src/topology_data.rs")) as fh:
        tpl = parse_templates(fh.read())
    assert sorted(tpl) == sorted(AA3), sorted(tpl)
    write_templates(tpl, os.path.join(HERE, "residue_templates.tbl"))

    with open(os.path.join(ref, "data/charmm36/par_all36m_prot.prm")) as fh:
        recs = parse_prm(fh.read())
    with open(os.path.join(ref, "data/charmm36/top_all36_prot.rtf")) as fh:
        charges = parse_rtf(fh.read(), tpl)
    lines = [
        "# CHARMM36m protein parameters (Huang & MacKerell 2016, par_all36m_prot.prm /",
        "# top_all36_prot.rtf, academic redistribution with attribution), reduced by",
        "# make_tables.py to the records origami's parser accepts for its atom types.",
        "# Units as in CHARMM: kcal/mol, Angstrom, degrees; NONBONDED epsilon is stored negative.",
    ]
    lines += recs
    for (aa, name), q in sorted(charges.items(), key=lambda kv: (AA3.index(kv[0][0]), kv[0][1])):
        if name:
            lines.append(f"CHARGE {aa} {name} {q}")
    with open(os.path.join(HERE, "charmm36m_protein.ff"), "w") as fh:
        fh.write("\n".join(lines) + "\n")
    print(f"templates: {sum(len(t['atoms']) for t in tpl.values())} side-chain atoms; "
          f"ff: {len(recs)} records, {len(charges)} charges")
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
