// CHARMM36m parameter tables and lookups.
//
// Insertion and lookup rules restate chem/src/forcefield.rs:
//   canonical_pair/triple/quad :160-179, bond/angle/dihedral/improper lookups
//   :84-158 (dihedral falls back to the X-b-c-X wildcard; improper tries each
//   atom as the central one, sorted off-atoms, then central+one-specific
//   wildcard), first-wins insertion for bonds/angles/impropers/nonbonded and
//   appended terms for dihedrals (parse_*_line :297-438), disulfide S-S patch
//   K = 173, r0 = 2.029 (:206).
#include <algorithm>
#include <fstream>
#include <sstream>

#include "model.h"

namespace og {

namespace {

std::pair<int, int> canon2(int a, int b) { return a <= b ? std::make_pair(a, b) : std::make_pair(b, a); }

std::tuple<int, int, int> canon3(int a, int b, int c) {
  return a <= c ? std::make_tuple(a, b, c) : std::make_tuple(c, b, a);
}

std::tuple<int, int, int, int> canon4(int a, int b, int c, int d) {
  // (b, a) <= (c, d) lexicographically keeps the order, else reverse.
  if (std::make_pair(b, a) <= std::make_pair(c, d)) return std::make_tuple(a, b, c, d);
  return std::make_tuple(d, c, b, a);
}

// Atom token: a modelled type index, -2 for the 'X' wildcard.
int tok_type(const std::string& t) {
  if (t == "X" || t == "x") return -2;
  return atom_type_from_name(t);
}

}  // namespace

std::string ForceField::load(const std::string& path) {
  std::ifstream in(path);
  if (!in) return "cannot open force-field table " + path;
  std::string line;
  int lineno = 0;
  while (std::getline(in, line)) {
    ++lineno;
    if (line.empty() || line[0] == '#') continue;
    std::istringstream ss(line);
    std::string kind;
    ss >> kind;
    auto bad = [&](const char* what) {
      return path + ":" + std::to_string(lineno) + ": bad " + what + " record";
    };
    if (kind == "BOND") {
      std::string a, b; double k, r0;
      if (!(ss >> a >> b >> k >> r0)) return bad("BOND");
      int ta = tok_type(a), tb = tok_type(b);
      if (ta < 0 || tb < 0) return bad("BOND");
      bonds_.emplace(canon2(ta, tb), BondParams{k, r0});
    } else if (kind == "ANGLE") {
      std::string a, b, c; double k, th;
      if (!(ss >> a >> b >> c >> k >> th)) return bad("ANGLE");
      int ta = tok_type(a), tb = tok_type(b), tc = tok_type(c);
      if (ta < 0 || tb < 0 || tc < 0) return bad("ANGLE");
      angles_.emplace(canon3(ta, tb, tc), AngleParams{k, th});
    } else if (kind == "DIHEDRAL") {
      std::string a, b, c, d; double k; int n; double delta;
      if (!(ss >> a >> b >> c >> d >> k >> n >> delta)) return bad("DIHEDRAL");
      int ta = tok_type(a), tb = tok_type(b), tc = tok_type(c), td = tok_type(d);
      DihedralTerm term{k, n, delta};
      if (ta >= 0 && tb >= 0 && tc >= 0 && td >= 0) {
        dihedrals_[canon4(ta, tb, tc, td)].push_back(term);
      } else if (ta == -2 && td == -2 && tb >= 0 && tc >= 0) {
        wildcard_dihedrals_[canon2(tb, tc)].push_back(term);
      } else {
        return bad("DIHEDRAL");
      }
    } else if (kind == "IMPROPER") {
      std::string a, b, c, d; double k, psi0;
      if (!(ss >> a >> b >> c >> d >> k >> psi0)) return bad("IMPROPER");
      int ta = tok_type(a), tb = tok_type(b), tc = tok_type(c), td = tok_type(d);
      ImproperParams p{k, psi0};
      if (ta >= 0 && tb == -2 && tc == -2 && td >= 0) {
        wildcard_impropers_.emplace(std::make_pair(ta, td), p);
      } else if (ta >= 0 && tb >= 0 && tc >= 0 && td >= 0) {
        int off[3] = {tb, tc, td};
        std::sort(off, off + 3);
        impropers_.emplace(std::make_tuple(off[0], ta, off[1], off[2]), p);
      } else {
        return bad("IMPROPER");
      }
    } else if (kind == "NONBONDED") {
      std::string t, e, r, e14, r14;
      if (!(ss >> t >> e >> r >> e14 >> r14)) return bad("NONBONDED");
      int tt = tok_type(t);
      if (tt < 0) return bad("NONBONDED");
      NonbondedParams p{};
      p.epsilon = -std::stod(e);
      p.rmin_half = std::stod(r);
      p.has14 = (e14 != "-");
      p.epsilon_14 = p.has14 ? -std::stod(e14) : 0.0;
      p.rmin_half_14 = p.has14 ? std::stod(r14) : 0.0;
      nonbonded_.emplace(tt, p);
    } else if (kind == "CHARGE") {
      std::string res, name; double q;
      if (!(ss >> res >> name >> q)) return bad("CHARGE");
      int aa = aa_from_three_letter(res);
      if (aa < 0) return bad("CHARGE");
      charges_[std::make_pair(aa, name)] = q;
    } else {
      return path + ":" + std::to_string(lineno) + ": unknown record " + kind;
    }
  }
  // Disulfide SG-SG bond (chem/src/forcefield.rs:206 patch_disulfide_bond).
  bonds_.emplace(canon2(T_S, T_S), BondParams{173.0, 2.029});
  if (bonds_.empty() || angles_.empty() || dihedrals_.empty() || nonbonded_.empty())
    return "force-field table " + path + " is incomplete";
  return "";
}

const BondParams* ForceField::bond(int a, int b) const {
  auto it = bonds_.find(canon2(a, b));
  return it == bonds_.end() ? nullptr : &it->second;
}

const AngleParams* ForceField::angle(int a, int b, int c) const {
  auto it = angles_.find(canon3(a, b, c));
  return it == angles_.end() ? nullptr : &it->second;
}

const std::vector<DihedralTerm>* ForceField::dihedral(int a, int b, int c, int d) const {
  auto it = dihedrals_.find(canon4(a, b, c, d));
  if (it != dihedrals_.end()) return &it->second;
  auto jt = wildcard_dihedrals_.find(canon2(b, c));
  return jt == wildcard_dihedrals_.end() ? nullptr : &jt->second;
}

const ImproperParams* ForceField::improper(int a, int b, int c, int d) const {
  const int all[4] = {a, b, c, d};
  const int centrals[4] = {b, a, c, d};
  for (int central : centrals) {
    int off[3];
    int k = 0;
    for (int t : all)
      if (t != central && k < 3) off[k++] = t;
    while (k < 3) off[k++] = central;
    std::sort(off, off + 3);
    auto it = impropers_.find(std::make_tuple(off[0], central, off[1], off[2]));
    if (it != impropers_.end()) return &it->second;
    for (int spec : off) {
      auto jt = wildcard_impropers_.find(std::make_pair(central, spec));
      if (jt != wildcard_impropers_.end()) return &jt->second;
    }
  }
  return nullptr;
}

const NonbondedParams* ForceField::nonbonded(int t) const {
  auto it = nonbonded_.find(t);
  return it == nonbonded_.end() ? nullptr : &it->second;
}

bool ForceField::partial_charge(int aa, const std::string& name, double* q) const {
  auto it = charges_.find(std::make_pair(aa, name));
  if (it == charges_.end()) return false;
  *q = it->second;
  return true;
}

}  // namespace og
