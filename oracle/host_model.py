"""Independent CPU restatement of origami's host model -- test infrastructure.

This is the checker for the product's C++ host model (atom typing, force-field
parameters, residue templates, topology graph, exclusions, per-atom caches,
SHAKE constraints).  It shares no code and no data file with the product: it
reads the reference's own Rust tables and CHARMM files from a reference
checkout and restates each rule from the reference's source.  Nothing in the
product imports it; tests/golden/make_host_golden.py runs it where a checkout
is present and commits its output as fixtures, which the CPU tests compare
with the product array by array.

Sources restated (paths relative to the reference's crates/ directory):
  classify                      chem/src/atom_type.rs:164-345 (match arms read
                                from the source, evaluated first-match-wins)
  AtomType order (Ord)          chem/src/atom_type.rs:6-58 (enum declaration)
  residue templates             chem/src/topology_data.rs (side-chain atoms,
                                bond_to parents, has_amide_h, is_glycine)
  .prm parser and lookups       chem/src/forcefield.rs:84-158 (lookups,
                                wildcards), :160-179 (canonical keys),
                                :218-436 (parser), :187-206 (SS patch)
  .rtf charges, name mapping    chem/src/forcefield.rs:444-599
  masses                        chem/src/element.rs:27-37
  GB rho / HCT scale            energy/src/gb.rs:58-83
  per-atom caches               energy/src/scratch.rs:196-230 (rebuild_params)
  topology graph                geom/src/topology_graph.rs:134-389
  exclusions / 1-4              energy/src/scratch.rs:233-251 with the graph
                                predicates of topology_graph.rs:81-112
  X-H constraints               dynamics/src/shake.rs:47-76
  builder atom order            geom/src/builder.rs:116-190
  PDB reader                    io/src/pdb_read.rs:163-462
"""
from __future__ import annotations

import os
import re
from dataclasses import dataclass, field

import numpy as np

AA_THREE = ["ALA", "ARG", "ASN", "ASP", "CYS", "GLN", "GLU", "GLY", "HIS", "ILE",
            "LEU", "LYS", "MET", "PHE", "PRO", "SER", "THR", "TRP", "TYR", "VAL"]
# IUPAC one-letter codes of AminoAcid::ALL (chem/src/amino_acid.rs:31)
AA_ONE = "ARNDCQEGHILKMFPSTWYV"
ELEMENTS = "HCNOPS"  # og_topology element codes 0..5
# element.rs:27-37
MASS = {"H": 1.008, "C": 12.011, "N": 14.007, "O": 15.999, "P": 30.974, "S": 32.06}
# gb.rs:58-68 and :73-83
GB_RHO = {"H": 1.20, "C": 1.70, "N": 1.55, "O": 1.50, "P": 1.85, "S": 1.80}
GB_SCALE = {"H": 0.85, "C": 0.72, "N": 0.79, "O": 0.85, "P": 0.86, "S": 0.96}
KIND_EXCLUDED, KIND_ONE_FOUR = 1, 2


def _strip_rust_comments(text: str) -> str:
    return re.sub(r"//[^\n]*", "", text)


def _read(ref: str, rel: str) -> str:
    with open(os.path.join(ref, rel)) as fh:
        return fh.read()


# ------------------------------------------------------------ atom typing
def parse_enum(text: str, name: str) -> list[str]:
    body = re.search(r"pub enum " + name + r"\s*\{(.*?)\}", _strip_rust_comments(text), re.S).group(1)
    return [t.strip() for t in body.split(",") if t.strip()]


@dataclass
class ClassifyArm:
    aa: str | None          # Rust AminoAcid variant, None = any
    names: set | None       # atom names, None = any
    result: str | None      # AtomType variant, None = not modelled


def parse_classify(text: str) -> list[ClassifyArm]:
    body = text[text.index("pub fn classify("):text.index("#[cfg(test)]")]
    body = _strip_rust_comments(body)
    arm = re.compile(r"\(\s*(\w+)\s*,\s*(_|(?:\"[A-Z0-9]+\"\s*\|?\s*)+)\)\s*=>\s*"
                     r"(return\s+Some\(\s*(\w+)\s*\)|return\s+None|(\w+))")
    arms = []
    for m in arm.finditer(body):
        aa = None if m.group(1) == "_" else m.group(1)
        names = None if m.group(2) == "_" else set(re.findall(r"\"([A-Z0-9]+)\"", m.group(2)))
        res = m.group(4) or m.group(5)
        arms.append(ClassifyArm(aa, names, res))
    return arms


# ------------------------------------------------------ residue templates
@dataclass
class SideAtom:
    name: str
    element: str
    bond_to: str


@dataclass
class Template:
    sidechain: list
    has_amide_h: bool
    is_glycine: bool


def parse_templates(text: str, aa_variants: list[str]) -> dict:
    src = _strip_rust_comments(text)
    const_of = dict(re.findall(r"AminoAcid::(\w+)\s*=>\s*&(\w+)", src))
    atom_re = re.compile(
        r"cb_atom\(\)"
        r"|(?:methyl_h|beta_h|ch2_chi)\(\s*\"(\w+)\"\s*,\s*\"(\w+)\""
        r"|SidechainAtom\s*\{\s*name:\s*\"(\w+)\"\s*,\s*element:\s*Element::(\w)\s*,\s*bond_to:\s*\"(\w+)\"")
    out = {}
    for var in aa_variants:
        const = const_of[var]
        m = re.search(r"const " + const + r": ResidueTopology = ResidueTopology \{(.*?)\n\};", src, re.S)
        block = m.group(1)
        side = block[block.index("sidechain:"):block.index("default_chi_rad:")]
        atoms = []
        for a in atom_re.finditer(side):
            if a.group(0) == "cb_atom()":
                # topology_data.rs:44-55: CB, carbon, bonded to CA
                atoms.append(SideAtom("CB", "C", "CA"))
            elif a.group(1):
                atoms.append(SideAtom(a.group(1), "H", a.group(2)))
            else:
                atoms.append(SideAtom(a.group(3), a.group(4), a.group(5)))
        has_h = re.search(r"has_amide_h:\s*(true|false)", block).group(1) == "true"
        is_gly = re.search(r"is_glycine:\s*(true|false)", block).group(1) == "true"
        out[var] = Template(atoms, has_h, is_gly)
    return out


# ------------------------------------------------------------ force field
@dataclass
class ForceField:
    types: list                     # AtomType variants in Ord order
    bonds: dict = field(default_factory=dict)
    angles: dict = field(default_factory=dict)
    dihedrals: dict = field(default_factory=dict)
    wildcard_dihedrals: dict = field(default_factory=dict)
    impropers: dict = field(default_factory=dict)
    wildcard_impropers: dict = field(default_factory=dict)
    nonbonded: dict = field(default_factory=dict)
    charges: dict = field(default_factory=dict)

    # forcefield.rs:160-179 -- keys compare by the enum's declaration order
    @staticmethod
    def pair(a, b):
        return (a, b) if a <= b else (b, a)

    @staticmethod
    def triple(a, b, c):
        return (a, b, c) if a <= c else (c, b, a)

    @staticmethod
    def quad(a, b, c, d):
        return (a, b, c, d) if (b, a) <= (c, d) else (d, c, b, a)

    # forcefield.rs:84-147
    def bond(self, a, b):
        return self.bonds.get(self.pair(a, b))

    def angle(self, a, b, c):
        return self.angles.get(self.triple(a, b, c))

    def dihedral(self, a, b, c, d):
        t = self.dihedrals.get(self.quad(a, b, c, d))
        if t is not None:
            return t
        return self.wildcard_dihedrals.get(self.pair(b, c))

    def improper(self, a, b, c, d):
        for central in (b, a, c, d):
            others = [t for t in (a, b, c, d) if t != central]
            while len(others) < 3:
                others.append(central)
            off = sorted(others[:3])
            p = self.impropers.get((off[0], central, off[1], off[2]))
            if p is not None:
                return p
            for spec in off:
                p = self.wildcard_impropers.get((central, spec))
                if p is not None:
                    return p
        return None


def _num(tok: str):
    try:
        return float(tok)
    except ValueError:
        return None


def parse_prm(text: str, types: list[str]) -> ForceField:
    ff = ForceField(types)
    index = {t: i for i, t in enumerate(types)}

    def atom(tok):
        if tok in ("X", "x"):
            return "X"
        return index.get(tok)

    section = None
    headers = {"BONDS": "bonds", "ANGLES": "angles", "DIHEDRALS": "dihedrals", "IMPROPER": "impropers",
               "IMPROPERS": "impropers", "CMAP": "cmap", "NONBONDED": "nonbonded", "HBOND": "hbond", "END": "end"}
    for raw in text.splitlines():
        line = raw.split("!", 1)[0].strip()
        if not line:
            continue
        first = line.split()[0]
        if first in headers:
            section = headers[first]
            if section == "end":
                break
            continue
        if section is None or section in ("cmap", "hbond"):
            continue
        tok = line.split()
        if section == "bonds" and len(tok) >= 4:
            a, b = atom(tok[0]), atom(tok[1])
            k, r0 = _num(tok[2]), _num(tok[3])
            if isinstance(a, int) and isinstance(b, int) and k is not None and r0 is not None:
                ff.bonds.setdefault(ff.pair(a, b), (k, r0))
        elif section == "angles" and len(tok) >= 5:
            a, b, c = atom(tok[0]), atom(tok[1]), atom(tok[2])
            k, th = _num(tok[3]), _num(tok[4])
            if all(isinstance(x, int) for x in (a, b, c)) and k is not None and th is not None:
                ff.angles.setdefault(ff.triple(a, b, c), (k, th))
        elif section == "dihedrals" and len(tok) >= 7:
            a, b, c, d = (atom(t) for t in tok[:4])
            k = _num(tok[4])
            n = int(tok[5]) if tok[5].isdigit() else None
            delta = _num(tok[6])
            if k is None or n is None or delta is None:
                continue
            if all(isinstance(x, int) for x in (a, b, c, d)):
                ff.dihedrals.setdefault(ff.quad(a, b, c, d), []).append((k, n, delta))
            elif a == "X" and d == "X" and isinstance(b, int) and isinstance(c, int):
                ff.wildcard_dihedrals.setdefault(ff.pair(b, c), []).append((k, n, delta))
        elif section == "impropers" and len(tok) >= 7:
            a, b, c, d = (atom(t) for t in tok[:4])
            k, psi0 = _num(tok[4]), _num(tok[6])
            if k is None or psi0 is None:
                continue
            if isinstance(a, int) and b == "X" and c == "X" and isinstance(d, int):
                ff.wildcard_impropers.setdefault((a, d), (k, psi0))
            elif all(isinstance(x, int) for x in (a, b, c, d)):
                off = sorted((b, c, d))
                ff.impropers.setdefault((off[0], a, off[1], off[2]), (k, psi0))
        elif section == "nonbonded":
            if "cutnb" in line or "ctofnb" in line or len(tok) < 4:
                continue
            t = atom(tok[0])
            eps, rmin = _num(tok[2]), _num(tok[3])
            if not isinstance(t, int) or eps is None or rmin is None:
                continue
            p = {"epsilon": -eps, "rmin_half": rmin, "epsilon_14": None, "rmin_half_14": None}
            if len(tok) >= 7:
                e14, r14 = _num(tok[5]), _num(tok[6])
                if e14 is not None and r14 is not None:
                    p["epsilon_14"], p["rmin_half_14"] = -e14, r14
            ff.nonbonded.setdefault(t, p)
    # forcefield.rs:187-206: SM-SM parameters on the S type, unless present
    s = index["S"]
    ff.bonds.setdefault(ff.pair(s, s), (173.0, 2.029))
    return ff


# forcefield.rs:520-577 -- CHARMM -> PDB v3.3 atom names, per residue
_B_SHIFT = {"Leu", "Met", "Pro", "Ser", "Cys", "Asn", "Gln", "Asp", "Glu", "Lys", "Arg", "His", "Phe", "Tyr", "Trp"}
_G_SHIFT = {"Met", "Pro", "Gln", "Glu", "Lys", "Arg"}
_D_SHIFT = {"Pro", "Lys", "Arg"}


def charmm_to_pdb(aa: str, name: str, templates: dict) -> str:
    if name == "HN":
        return "H"
    fixed = {("Gly", "HA1"): "HA2", ("Gly", "HA2"): "HA3",
             ("Ile", "CD"): "CD1", ("Ile", "HD1"): "HD11", ("Ile", "HD2"): "HD12", ("Ile", "HD3"): "HD13",
             ("Ile", "HG11"): "HG12", ("Ile", "HG12"): "HG13",
             ("Ser", "HG1"): "HG", ("Cys", "HG1"): "HG",
             ("Lys", "HE1"): "HE2", ("Lys", "HE2"): "HE3"}
    if (aa, name) in fixed:
        return fixed[(aa, name)]
    for group, base in ((_B_SHIFT, "HB"), (_G_SHIFT, "HG"), (_D_SHIFT, "HD")):
        if aa in group and name in (base + "1", base + "2"):
            return base + ("2" if name.endswith("1") else "3")
    if name in ("N", "CA", "C", "O", "HA"):
        return name
    for sc in templates[aa].sidechain:
        if sc.name == name:
            return name
    return ""


def parse_rtf(text: str, ff: ForceField, templates: dict) -> None:
    resi = {"ALA": "Ala", "ARG": "Arg", "ASN": "Asn", "ASP": "Asp", "CYS": "Cys", "GLN": "Gln", "GLU": "Glu",
            "GLY": "Gly", "HSD": "His", "ILE": "Ile", "LEU": "Leu", "LYS": "Lys", "MET": "Met", "PHE": "Phe",
            "PRO": "Pro", "SER": "Ser", "THR": "Thr", "TRP": "Trp", "TYR": "Tyr", "VAL": "Val"}
    current = None
    for raw in text.splitlines():
        line = raw.split("!", 1)[0].strip()
        if not line:
            continue
        tok = line.split()
        if tok[0] == "RESI":
            current = resi.get(tok[1] if len(tok) > 1 else "")
            continue
        if tok[0] == "PRES":
            current = None
            continue
        if tok[0] != "ATOM" or current is None or len(tok) < 4:
            continue
        q = _num(tok[3])
        if q is None:
            continue
        ff.charges[(current, charmm_to_pdb(current, tok[1], templates))] = q


# ------------------------------------------------------------- the model
class HostModel:
    """The reference's host model, loaded from a reference checkout."""

    def __init__(self, ref: str):
        at = _read(ref, "crates/chem/src/atom_type.rs")
        aa = _read(ref, "crates/chem/src/amino_acid.rs")
        self.types = parse_enum(at, "AtomType")
        self.aa_variants = parse_enum(aa, "AminoAcid")
        assert [v.upper() for v in self.aa_variants] == AA_THREE
        self.arms = parse_classify(at)
        self.templates = parse_templates(_read(ref, "crates/chem/src/topology_data.rs"), self.aa_variants)
        self.ff = parse_prm(_read(ref, "data/charmm36/par_all36m_prot.prm"), self.types)
        parse_rtf(_read(ref, "data/charmm36/top_all36_prot.rtf"), self.ff, self.templates)

    def classify(self, aa: str, name: str):
        for arm in self.arms:
            if (arm.aa is None or arm.aa == aa) and (arm.names is None or name in arm.names):
                return None if arm.result is None else self.types.index(arm.result)
        return None

    def residue_atoms(self, aa: str, first: bool = False) -> list:
        """Atom names and elements of one built residue in builder order
        (builder.rs:116-190): N, CA, C, O, H, HA (HA2, HA3), side chain."""
        t = self.templates[aa]
        out = [("N", "N"), ("CA", "C"), ("C", "C"), ("O", "O")]
        if t.has_amide_h:
            out.append(("H", "H"))
        out += [("HA2", "H"), ("HA3", "H")] if t.is_glycine else [("HA", "H")]
        out += [(a.name, a.element) for a in t.sidechain]
        return out

    # topology_graph.rs:134-389
    def topology_graph(self, residues: list) -> dict:
        """residues: list of (aa variant, chain id, [(name, element, xyz)])."""
        idx = {}
        total = 0
        for ri, (_, _, atoms) in enumerate(residues):
            for name, _, _ in atoms:
                idx[(ri, name)] = total
                total += 1
        look = lambda ri, n: idx.get((ri, n))  # noqa: E731
        bonds = set()

        def add(a, b):
            if a is not None and b is not None and a != b:
                bonds.add((min(a, b), max(a, b)))

        rings = {"Pro": [("N", "CD")], "Phe": [("CE2", "CZ")], "Tyr": [("CE2", "CZ")], "His": [("CE1", "NE2")],
                 "Trp": [("CE2", "CD2"), ("CH2", "CZ3")]}
        for ri, (aa, chain, _) in enumerate(residues):
            n, ca, c, o = look(ri, "N"), look(ri, "CA"), look(ri, "C"), look(ri, "O")
            add(n, ca)
            add(ca, c)
            add(c, o)
            add(n, look(ri, "H"))
            if aa == "Gly":
                add(ca, look(ri, "HA2"))
                add(ca, look(ri, "HA3"))
            else:
                add(ca, look(ri, "HA"))
            if ri > 0 and residues[ri - 1][1] == chain:
                add(look(ri - 1, "C"), n)
            for sc in self.templates[aa].sidechain:
                add(look(ri, sc.bond_to), look(ri, sc.name))
            for a, b in rings.get(aa, []):
                add(look(ri, a), look(ri, b))
        sg = []
        for ri, (aa, _, atoms) in enumerate(residues):
            if aa != "Cys":
                continue
            for name, _, xyz in atoms:
                if name == "SG":
                    sg.append((look(ri, "SG"), np.asarray(xyz, dtype=np.float64)))
                    break
        for i in range(len(sg)):
            for j in range(i + 1, len(sg)):
                d = sg[i][1] - sg[j][1]
                if float(d @ d) <= 2.5 * 2.5:
                    add(sg[i][0], sg[j][0])
        bonds = sorted(bonds)
        nbr = [[] for _ in range(total)]
        for a, b in bonds:
            nbr[a].append(b)
            nbr[b].append(a)
        for v in nbr:
            v.sort()
        angles = [(v[i], b, v[j]) for b, v in enumerate(nbr) for i in range(len(v)) for j in range(i + 1, len(v))]
        seen, dihedrals = set(), []
        for b, c in bonds:
            for a in nbr[b]:
                if a == c:
                    continue
                for d in nbr[c]:
                    if d == b or d == a:
                        continue
                    key = (a, b, c, d) if b < c else (d, c, b, a)
                    if key not in seen:
                        seen.add(key)
                        dihedrals.append(key)
        impropers = []
        # (substituent, centre, substituent, substituent) as looked up;
        # stored centre first (topology_graph.rs:300-375)
        centres = {"Asn": ("CB", "CG", "OD1", "ND2"), "Gln": ("CG", "CD", "OE1", "NE2"),
                   "Asp": ("CB", "CG", "OD1", "OD2"), "Glu": ("CG", "CD", "OE1", "OE2"),
                   "Arg": ("NE", "CZ", "NH1", "NH2")}
        for ri, (aa, _, _) in enumerate(residues):
            if ri + 1 < len(residues):
                q = (look(ri, "CA"), look(ri, "C"), look(ri, "O"), look(ri + 1, "N"))
                if None not in q:
                    impropers.append((q[1], q[0], q[2], q[3]))
            if aa in centres:
                s, cen, p, r = centres[aa]
                q = (look(ri, s), look(ri, cen), look(ri, p), look(ri, r))
                if None not in q:
                    impropers.append((q[1], q[0], q[2], q[3]))
        return {"n": total, "bonds": bonds, "angles": angles, "dihedrals": dihedrals, "impropers": impropers,
                "nbr": nbr}

    @staticmethod
    def exclusions(g: dict) -> list:
        """scratch.rs:233-251 over topology_graph.rs:81-112."""
        nbr = [set(v) for v in g["nbr"]]
        out = []
        for i in range(g["n"]):
            one_two = nbr[i]
            one_three = set()
            for m in nbr[i]:
                one_three |= nbr[m]
            one_three.discard(i)
            one_four = set()
            for m in nbr[i]:
                for k in nbr[m]:
                    one_four |= nbr[k]
            for j in sorted(one_two | one_three | one_four):
                if j <= i:
                    continue
                if j in one_two or j in one_three:
                    out.append((i, j, KIND_EXCLUDED))
                else:
                    out.append((i, j, KIND_ONE_FOUR))
        return out

    def topology(self, residues: list) -> dict:
        """The og_topology arrays the reference's caches and graph amount to."""
        n = sum(len(a) for _, _, a in residues)
        charge, rmin, eps, rmin14, eps14 = (np.zeros(n) for _ in range(5))
        rho, scale, mass = (np.zeros(n) for _ in range(3))
        element = np.zeros(n, dtype=np.int32)
        types = np.zeros(n, dtype=np.int64)
        k = 0
        for aa, _, atoms in residues:
            for name, el, _ in atoms:
                t = self.classify(aa, name)
                if t is None:
                    raise ValueError(f"unclassified atom {aa} {name}")
                types[k] = t
                charge[k] = self.ff.charges.get((aa, name), 0.0)
                rho[k], scale[k], mass[k] = GB_RHO[el], GB_SCALE[el], MASS[el]
                element[k] = ELEMENTS.index(el)
                p = self.ff.nonbonded.get(t)
                if p is not None:
                    rmin[k], eps[k] = p["rmin_half"], p["epsilon"]
                    rmin14[k] = p["rmin_half"] if p["rmin_half_14"] is None else p["rmin_half_14"]
                    eps14[k] = p["epsilon"] if p["epsilon_14"] is None else p["epsilon_14"]
                k += 1
        g = self.topology_graph(residues)
        out = {"charge": charge, "rmin_half": rmin, "epsilon": eps, "rmin_half_14": rmin14, "epsilon_14": eps14,
               "gb_rho": rho, "gb_scale": scale, "mass": mass, "element": element, "atom_type": types}
        bonds, bk, br0, cons, clen = [], [], [], [], []
        for a, b in g["bonds"]:
            p = self.ff.bond(types[a], types[b])
            if p is None:
                continue
            bonds.append((a, b))
            bk.append(p[0])
            br0.append(p[1])
            if element[a] == 0 or element[b] == 0:  # shake.rs:57-72
                cons.append((a, b))
                clen.append(p[1])
        angles, ak, at0 = [], [], []
        for a, b, c in g["angles"]:
            p = self.ff.angle(types[a], types[b], types[c])
            if p is None:
                continue
            angles.append((a, b, c))
            ak.append(p[0])
            at0.append(p[1])
        dih, start, tk, tn, td = [], [0], [], [], []
        for q in g["dihedrals"]:
            terms = self.ff.dihedral(*(types[i] for i in q))
            if terms is None:
                continue
            dih.append(q)
            for kk, nn, dd in terms:
                tk.append(kk)
                tn.append(nn)
                td.append(dd)
            start.append(len(tk))
        imp, ik, ip0 = [], [], []
        for q in g["impropers"]:
            p = self.ff.improper(*(types[i] for i in q))
            if p is None:
                continue
            imp.append(q)
            ik.append(p[0])
            ip0.append(p[1])
        ex = self.exclusions(g)
        i32 = lambda v, w: np.asarray(v, dtype=np.int32).reshape(-1, w)  # noqa: E731
        out.update({
            "bonds": i32(bonds, 2), "bond_k": np.asarray(bk), "bond_r0": np.asarray(br0),
            "angles": i32(angles, 3), "angle_k": np.asarray(ak), "angle_theta0": np.asarray(at0),
            "dihedrals": i32(dih, 4), "dihedral_term_start": np.asarray(start, dtype=np.int32),
            "term_k": np.asarray(tk), "term_n": np.asarray(tn, dtype=np.int32), "term_delta": np.asarray(td),
            "impropers": i32(imp, 4), "improper_k": np.asarray(ik), "improper_psi0": np.asarray(ip0),
            "exclusions": i32([(i, j) for i, j, _ in ex], 2),
            "exclusion_kind": np.asarray([kk for _, _, kk in ex], dtype=np.int8),
            "constraints": i32(cons, 2), "constraint_length": np.asarray(clen),
        })
        return out


# ----------------------------------------------------------- PDB reading
_TERMINAL = {"H1", "H2", "H3", "OXT", "HXT"}
# nucleotide.rs:94-102: residue names skipped as RNA/DNA
_NUCLEOTIDES = {"A", "RA", "DA", "U", "RU", "T", "DT", "G", "RG", "DG", "C", "RC", "DC"}


def read_pdb(text: str, model: HostModel) -> list:
    """First model of a PDB file as (aa variant, chain id, [(name, element,
    xyz)]) residues: pdb_read.rs:163-272 (records, alternate locations,
    residue grouping by chain and sequence number, first occurrence of a
    name wins) with :347-462 (name normalisation, canonical names, terminal
    atoms skipped, element from columns 77-78 or the name)."""
    three = {a: v for a, v in zip(AA_THREE, model.aa_variants)}
    residues, current, found = [], None, False
    for lineno, line in enumerate(text.splitlines(), 1):
        if line.startswith("END"):
            if residues:
                break
            continue
        if line.startswith("MODEL") and residues:
            break
        if line.startswith("TER") or not line.startswith("ATOM"):
            continue
        s = line.ljust(80)
        name, alt, resn, chain = s[12:16].strip(), s[16], s[17:20].strip(), s[21]
        seq = int(s[22:26].strip())
        xyz = (float(s[30:38]), float(s[38:46]), float(s[46:54]))
        el_col = s[76:78].strip().upper()
        if alt not in (" ", "A"):
            continue
        aa = three.get(resn.upper()) if len(resn) == 3 else None
        if aa is None:
            if resn in _NUCLEOTIDES:
                continue
            raise ValueError(f"line {lineno}: unknown residue {resn}")
        if len(name) >= 4 and name[0].isdigit():
            name = name[1:] + name[0]
        canon = None
        if name in ("N", "CA", "C", "O", "H", "HA", "HA2", "HA3"):
            canon = name
        elif name not in ("OXT", "H1", "H2", "H3"):
            for sc in model.templates[aa].sidechain:
                if sc.name == name:
                    canon = name
                    break
        if canon is None:
            if name in _TERMINAL:
                continue
            raise ValueError(f"line {lineno}: atom {name} not part of {aa}")
        el = el_col if el_col in MASS and el_col != "P" else None
        if el is None:
            el = canon[0] if canon[0] in "HCNOS" else None
            if el is None:
                raise ValueError(f"line {lineno}: no element for {canon}")
        key = (chain, seq)
        if key != current:
            residues.append([aa, chain, [], set()])
            current = key
        r = residues[-1]
        if canon not in r[3]:
            r[3].add(canon)
            r[2].append((canon, el, xyz))
        found = True
    if not found:
        raise ValueError("no ATOM records")
    return [(aa, ch, atoms) for aa, ch, atoms, _ in residues]
