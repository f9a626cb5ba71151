// Residue templates and the NeRF chain builder.
//
// place_atom restates geom/src/nerf.rs:15-36; append_residue restates
// geom/src/builder.rs:78-238 (backbone anchor of the first residue, peptide
// placement of N/CA/C by psi/omega/phi, O at psi+pi, amide H, HA / HA2+HA3,
// then the side-chain template atoms in table order).
#include <cmath>
#include <fstream>
#include <sstream>

#include "model.h"

namespace og {

const double kDefaultPhi = -120.0 * M_PI / 180.0;
const double kDefaultPsi = 140.0 * M_PI / 180.0;
const double kDefaultOmega = M_PI;

namespace {
constexpr double kCbDihedral = -122.55 * M_PI / 180.0;
constexpr double kPeptideCN = 1.329;
constexpr double kNCa = 1.458;
constexpr double kCaC = 1.525;
constexpr double kCO = 1.231;
constexpr double kNHAmide = 1.010;
constexpr double kCaHa = 1.090;
constexpr double kCNCaAngle = 121.7 * M_PI / 180.0;
constexpr double kCaCOAngle = 120.8 * M_PI / 180.0;
constexpr double kHnBondAngle = 119.0 * M_PI / 180.0;
constexpr double kHaBondAngle = 109.0 * M_PI / 180.0;
constexpr double kNCaCAngle = 111.2 * M_PI / 180.0;   // chem topology angle::N_CA_C
constexpr double kCaCNAngle = 116.2 * M_PI / 180.0;   // chem topology angle::CA_C_N

Vec3 sub(Vec3 a, Vec3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
Vec3 add(Vec3 a, Vec3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
Vec3 scale(Vec3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
Vec3 cross(Vec3 a, Vec3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
Vec3 normalize(Vec3 a) {
  double n = std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z);
  return {a.x / n, a.y / n, a.z / n};
}

bool find_pos(const PlacedResidue& r, const std::string& name, Vec3* out) {
  for (const auto& a : r.atoms)
    if (a.name == name) { *out = a.pos; return true; }
  return false;
}
}  // namespace

int Structure::atom_count() const {
  int n = 0;
  for (const auto& r : residues) n += static_cast<int>(r.atoms.size());
  return n;
}

Vec3 place_atom(Vec3 a, Vec3 b, Vec3 c, double length, double angle, double dihedral) {
  Vec3 bc = normalize(sub(c, b));
  Vec3 ba = sub(a, b);
  Vec3 n = normalize(cross(bc, ba));
  Vec3 x_hat = bc, z_hat = n;
  Vec3 y_hat = cross(z_hat, x_hat);
  double sin_t = std::sin(angle), cos_t = std::cos(angle);
  double sin_d = std::sin(dihedral), cos_d = std::cos(dihedral);
  // offset = -x*(L cos t) + y*(L sin t cos d) + z*(L sin t sin d), summed left to right
  Vec3 off = add(add(scale(x_hat, -(length * cos_t)), scale(y_hat, length * sin_t * cos_d)),
                 scale(z_hat, length * sin_t * sin_d));
  return add(c, off);
}

std::string Templates::load(const std::string& path) {
  std::ifstream in(path);
  if (!in) return "cannot open residue-template table " + path;
  std::string line;
  int cur = -1;
  int lineno = 0;
  while (std::getline(in, line)) {
    ++lineno;
    if (line.empty() || line[0] == '#') continue;
    std::istringstream ss(line);
    std::string kind;
    ss >> kind;
    if (kind == "RES") {
      std::string name; int amide, gly, nchi;
      if (!(ss >> name >> amide >> gly >> nchi)) return path + ":" + std::to_string(lineno) + ": bad RES";
      cur = aa_from_three_letter(name);
      if (cur < 0) return path + ": unknown residue " + name;
      ResidueTemplate& t = res_[cur];
      t = ResidueTemplate{};
      t.has_amide_h = amide != 0;
      t.is_glycine = gly != 0;
      for (int i = 0; i < nchi; ++i) {
        double v;
        if (!(ss >> v)) return path + ":" + std::to_string(lineno) + ": bad chi list";
        t.default_chi.push_back(v);
      }
    } else if (kind == "ATOM") {
      if (cur < 0) return path + ": ATOM before RES";
      TemplateAtom a;
      std::string el, kd;
      if (!(ss >> a.name >> el >> a.bond_to >> a.angle_at >> a.dihedral_to >> a.bond_length >>
            a.bond_angle >> kd >> a.chi_n >> a.value))
        return path + ":" + std::to_string(lineno) + ": bad ATOM";
      if (!element_from_symbol(el, &a.element)) return path + ": bad element " + el;
      a.kind = kd[0];
      res_[cur].sidechain.push_back(a);
    } else {
      return path + ":" + std::to_string(lineno) + ": unknown record " + kind;
    }
  }
  return "";
}

std::string append_residue(Structure* s, const Templates& tpl, int aa, double phi, double psi,
                           double omega) {
  if (aa < 0 || aa >= kNumAminoAcids) return "unknown amino acid";
  const ResidueTemplate& topo = tpl.get(aa);
  const size_t idx = s->residues.size();
  PlacedResidue res{aa, 'A', {}};
  Vec3 n_pos, ca_pos, c_pos;
  if (idx == 0) {
    n_pos = {0.0, 0.0, 0.0};
    ca_pos = {kNCa, 0.0, 0.0};
    double dx = -kCaC * std::cos(kNCaCAngle);
    double dy = kCaC * std::sin(kNCaCAngle);
    c_pos = {ca_pos.x + dx, ca_pos.y + dy, 0.0};
  } else {
    const PlacedResidue& prev = s->residues[idx - 1];
    Vec3 pn, pca, pc;
    find_pos(prev, "N", &pn);
    find_pos(prev, "CA", &pca);
    find_pos(prev, "C", &pc);
    n_pos = place_atom(pn, pca, pc, kPeptideCN, kCaCNAngle, psi);
    ca_pos = place_atom(pca, pc, n_pos, kNCa, kCNCaAngle, omega);
    c_pos = place_atom(pc, n_pos, ca_pos, kCaC, kNCaCAngle, phi);
  }
  res.atoms.push_back({"N", Element::N, n_pos});
  res.atoms.push_back({"CA", Element::C, ca_pos});
  res.atoms.push_back({"C", Element::C, c_pos});
  Vec3 o = place_atom(n_pos, ca_pos, c_pos, kCO, kCaCOAngle, psi + M_PI);
  res.atoms.push_back({"O", Element::O, o});

  if (topo.has_amide_h && idx > 0) {
    const PlacedResidue& prev = s->residues[idx - 1];
    Vec3 pc, po;
    find_pos(prev, "C", &pc);
    find_pos(prev, "O", &po);
    res.atoms.push_back({"H", Element::H, place_atom(po, pc, n_pos, kNHAmide, kHnBondAngle, M_PI)});
  } else if (topo.has_amide_h && idx == 0) {
    res.atoms.push_back({"H", Element::H, place_atom(c_pos, ca_pos, n_pos, kNHAmide, kHnBondAngle, M_PI)});
  }

  if (topo.is_glycine) {
    res.atoms.push_back({"HA2", Element::H, place_atom(c_pos, n_pos, ca_pos, kCaHa, kHaBondAngle, -kCbDihedral)});
    res.atoms.push_back({"HA3", Element::H, place_atom(c_pos, n_pos, ca_pos, kCaHa, kHaBondAngle, kCbDihedral)});
  } else {
    res.atoms.push_back({"HA", Element::H, place_atom(c_pos, n_pos, ca_pos, kCaHa, kHaBondAngle, -kCbDihedral)});
  }

  auto lookup = [&](const std::string& name, Vec3* out) -> bool {
    if (find_pos(res, name, out)) return true;
    if (idx > 0 && find_pos(s->residues[idx - 1], name, out)) return true;
    return false;
  };
  for (const TemplateAtom& t : topo.sidechain) {
    Vec3 pa, pb, pc;
    if (!lookup(t.dihedral_to, &pa) || !lookup(t.angle_at, &pb) || !lookup(t.bond_to, &pc))
      return std::string("residue ") + std::to_string(idx) + " references an unplaced atom";
    double dih = t.value;
    if (t.kind == 'C') dih = topo.default_chi[t.chi_n - 1];
    else if (t.kind == 'P') dih = topo.default_chi[t.chi_n - 1] + t.value;
    res.atoms.push_back({t.name, t.element, place_atom(pa, pb, pc, t.bond_length, t.bond_angle, dih)});
  }
  s->residues.push_back(std::move(res));
  return "";
}

}  // namespace og
