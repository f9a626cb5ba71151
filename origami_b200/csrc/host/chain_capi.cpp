// og_chain_*: the sequence -> flat og_topology half of the C ABI.
//
// Per-atom parameters follow ForceScratch::rebuild_params
// (energy/src/scratch.rs:196-230): classify -> CHARMM type, partial charge
// from the .rtf table (0 when absent), GB rho / rho-tilde / HCT scale from the
// element (energy/src/gb.rs:58-83), LJ params with the 1-4 values falling back
// to the regular ones.  Bonded terms carry the parameters origami's force code
// looks up per call (energy/src/forces_bonded.rs); X-H constraints follow
// dynamics/src/shake.rs:47-76.
#include <dlfcn.h>

#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>

#include "../../../include/origami_gpu.h"
#include "chain.h"
#include "model.h"
#include "status.h"

namespace {

std::mutex g_data_mu;
std::string g_data_dir;
std::unique_ptr<og::ForceField> g_ff;
std::unique_ptr<og::Templates> g_tpl;

std::string default_data_dir() {
  Dl_info info;
  if (dladdr(reinterpret_cast<void*>(&default_data_dir), &info) && info.dli_fname) {
    std::string p(info.dli_fname);
    size_t slash = p.rfind('/');
    return (slash == std::string::npos ? std::string(".") : p.substr(0, slash)) + "/data";
  }
  return "data";
}

og_status ensure_tables(const og::ForceField** ff, const og::Templates** tpl) {
  std::lock_guard<std::mutex> lock(g_data_mu);
  if (!g_ff) {
    std::string dir = g_data_dir.empty() ? default_data_dir() : g_data_dir;
    auto f = std::make_unique<og::ForceField>();
    std::string err = f->load(dir + "/charmm36m_protein.ff");
    if (!err.empty()) return og_fail(OG_E_DATA, err);
    auto t = std::make_unique<og::Templates>();
    err = t->load(dir + "/residue_templates.tbl");
    if (!err.empty()) return og_fail(OG_E_DATA, err);
    g_ff = std::move(f);
    g_tpl = std::move(t);
  }
  *ff = g_ff.get();
  *tpl = g_tpl.get();
  return OG_OK;
}

double gb_intrinsic_radius(og::Element e) {  // energy/src/gb.rs:58-68
  switch (e) {
    case og::Element::H: return 1.20;
    case og::Element::C: return 1.70;
    case og::Element::N: return 1.55;
    case og::Element::O: return 1.50;
    case og::Element::P: return 1.85;
    case og::Element::S: return 1.80;
  }
  return 0.0;
}

double gb_hct_scale(og::Element e) {  // energy/src/gb.rs:73-83
  switch (e) {
    case og::Element::H: return 0.85;
    case og::Element::C: return 0.72;
    case og::Element::N: return 0.79;
    case og::Element::O: return 0.85;
    case og::Element::P: return 0.86;
    case og::Element::S: return 0.96;
  }
  return 0.0;
}

}  // namespace

namespace {

og_status rebuild(og_chain* c) {
  const og::ForceField* ff;
  const og::Templates* tpl;
  og_status st = ensure_tables(&ff, &tpl);
  if (st != OG_OK) return st;
  const int n = c->s.atom_count();
  c->charge.assign(n, 0.0); c->rmin.assign(n, 0.0); c->eps.assign(n, 0.0);
  c->rmin14.assign(n, 0.0); c->eps14.assign(n, 0.0); c->rho.assign(n, 0.0);
  c->scale.assign(n, 0.0); c->mass.assign(n, 0.0);
  c->element.assign(n, 0); c->atom_type.assign(n, 0); c->residue_of.assign(n, 0);
  int idx = 0;
  for (size_t r = 0; r < c->s.residues.size(); ++r) {
    const auto& res = c->s.residues[r];
    for (const auto& a : res.atoms) {
      int t = og::classify(res.aa, a.name);
      if (t < 0) return og_fail(OG_E_DATA, std::string("unclassified atom ") + og::aa_three_letter(res.aa) + " " + a.name);
      c->atom_type[idx] = t;
      c->residue_of[idx] = static_cast<int32_t>(r);
      c->element[idx] = static_cast<int32_t>(a.element);
      double q = 0.0;
      ff->partial_charge(res.aa, a.name, &q);
      c->charge[idx] = q;
      c->rho[idx] = gb_intrinsic_radius(a.element);
      c->scale[idx] = gb_hct_scale(a.element);
      c->mass[idx] = og::element_mass(a.element);
      if (const og::NonbondedParams* p = ff->nonbonded(t)) {
        c->rmin[idx] = p->rmin_half;
        c->eps[idx] = p->epsilon;
        c->rmin14[idx] = p->has14 ? p->rmin_half_14 : p->rmin_half;
        c->eps14[idx] = p->has14 ? p->epsilon_14 : p->epsilon;
      }
      ++idx;
    }
  }
  og::Topology g = og::build_topology(c->s, *tpl);
  c->missing = 0;
  c->bond_atoms.clear(); c->bond_k.clear(); c->bond_r0.clear();
  c->cons_atoms.clear(); c->cons_d.clear();
  for (const auto& b : g.bonds) {
    const og::BondParams* p = ff->bond(c->atom_type[b[0]], c->atom_type[b[1]]);
    if (!p) { ++c->missing; continue; }
    c->bond_atoms.push_back(b[0]); c->bond_atoms.push_back(b[1]);
    c->bond_k.push_back(p->k); c->bond_r0.push_back(p->r0);
    const bool xh = c->element[b[0]] == 0 || c->element[b[1]] == 0;
    if (xh) {
      c->cons_atoms.push_back(b[0]); c->cons_atoms.push_back(b[1]);
      c->cons_d.push_back(p->r0);
    }
  }
  c->angle_atoms.clear(); c->angle_k.clear(); c->angle_t0.clear();
  for (const auto& a : g.angles) {
    const og::AngleParams* p = ff->angle(c->atom_type[a[0]], c->atom_type[a[1]], c->atom_type[a[2]]);
    if (!p) { ++c->missing; continue; }
    for (int k = 0; k < 3; ++k) c->angle_atoms.push_back(a[k]);
    c->angle_k.push_back(p->k); c->angle_t0.push_back(p->theta0_deg);
  }
  c->dih_atoms.clear(); c->dih_start.assign(1, 0); c->term_k.clear(); c->term_n.clear(); c->term_delta.clear();
  for (const auto& d : g.dihedrals) {
    const auto* terms = ff->dihedral(c->atom_type[d[0]], c->atom_type[d[1]], c->atom_type[d[2]], c->atom_type[d[3]]);
    if (!terms) { ++c->missing; continue; }
    for (int k = 0; k < 4; ++k) c->dih_atoms.push_back(d[k]);
    for (const auto& t : *terms) {
      c->term_k.push_back(t.k); c->term_n.push_back(t.n); c->term_delta.push_back(t.delta_deg);
    }
    c->dih_start.push_back(static_cast<int32_t>(c->term_k.size()));
  }
  c->imp_atoms.clear(); c->imp_k.clear(); c->imp_psi0.clear();
  for (const auto& im : g.impropers) {
    const og::ImproperParams* p = ff->improper(c->atom_type[im[0]], c->atom_type[im[1]], c->atom_type[im[2]], c->atom_type[im[3]]);
    if (!p) { ++c->missing; continue; }
    for (int k = 0; k < 4; ++k) c->imp_atoms.push_back(im[k]);
    c->imp_k.push_back(p->k); c->imp_psi0.push_back(p->psi0_deg);
  }
  auto ex = og::build_exclusions(g, n);
  c->excl_atoms.clear(); c->excl_kind.clear();
  for (const auto& e : ex) {
    c->excl_atoms.push_back(e.i); c->excl_atoms.push_back(e.j); c->excl_kind.push_back(e.kind);
  }

  og_topology& t = c->topo;
  t = og_topology{};
  t.n_atoms = n;
  t.charge = c->charge.data(); t.rmin_half = c->rmin.data(); t.epsilon = c->eps.data();
  t.rmin_half_14 = c->rmin14.data(); t.epsilon_14 = c->eps14.data();
  t.gb_rho = c->rho.data(); t.gb_scale = c->scale.data(); t.mass = c->mass.data();
  t.element = c->element.data();
  t.n_bonds = static_cast<int32_t>(c->bond_k.size());
  t.bond_atoms = c->bond_atoms.data(); t.bond_k = c->bond_k.data(); t.bond_r0 = c->bond_r0.data();
  t.n_angles = static_cast<int32_t>(c->angle_k.size());
  t.angle_atoms = c->angle_atoms.data(); t.angle_k = c->angle_k.data(); t.angle_theta0 = c->angle_t0.data();
  t.n_dihedrals = static_cast<int32_t>(c->dih_start.size()) - 1;
  t.dihedral_atoms = c->dih_atoms.data(); t.dihedral_term_start = c->dih_start.data();
  t.n_dihedral_terms = static_cast<int32_t>(c->term_k.size());
  t.term_k = c->term_k.data(); t.term_n = c->term_n.data(); t.term_delta = c->term_delta.data();
  t.n_impropers = static_cast<int32_t>(c->imp_k.size());
  t.improper_atoms = c->imp_atoms.data(); t.improper_k = c->imp_k.data(); t.improper_psi0 = c->imp_psi0.data();
  t.n_exclusions = static_cast<int32_t>(c->excl_kind.size());
  t.exclusion_atoms = c->excl_atoms.data(); t.exclusion_kind = c->excl_kind.data();
  t.n_constraints = static_cast<int32_t>(c->cons_d.size());
  t.constraint_atoms = c->cons_atoms.data(); t.constraint_length = c->cons_d.data();
  c->dirty = false;
  return OG_OK;
}

double or_default(double v, double d) { return std::isnan(v) ? d : v; }

}  // namespace

extern "C" {

og_status og_set_data_dir(const char* path) {
  if (!path) return og_fail(OG_E_BADARG, "null data dir");
  std::lock_guard<std::mutex> lock(g_data_mu);
  g_data_dir = path;
  g_ff.reset();
  g_tpl.reset();
  return OG_OK;
}

og_status og_chain_build(const char* sequence, double phi, double psi, double omega, og_chain** out) {
  if (!sequence || !out) return og_fail(OG_E_BADARG, "null argument");
  *out = nullptr;
  if (!*sequence) return og_fail(OG_E_BADARG, "empty sequence");
  const og::ForceField* ff;
  const og::Templates* tpl;
  og_status st = ensure_tables(&ff, &tpl);
  if (st != OG_OK) return st;
  auto c = std::make_unique<og_chain>();
  for (const char* p = sequence; *p; ++p) {
    int aa = og::aa_from_one_letter(*p);
    if (aa < 0) return og_fail(OG_E_BADARG, std::string("not an amino-acid code: ") + *p);
    std::string err = og::append_residue(&c->s, *tpl, aa, or_default(phi, og::kDefaultPhi),
                                         or_default(psi, og::kDefaultPsi), or_default(omega, og::kDefaultOmega));
    if (!err.empty()) return og_fail(OG_E_DATA, err);
  }
  st = rebuild(c.get());
  if (st != OG_OK) return st;
  *out = c.release();
  return OG_OK;
}

og_status og_chain_append(og_chain* c, char residue, double phi, double psi, double omega) {
  if (!c) return og_fail(OG_E_BADARG, "null chain");
  const og::ForceField* ff;
  const og::Templates* tpl;
  og_status st = ensure_tables(&ff, &tpl);
  if (st != OG_OK) return st;
  int aa = og::aa_from_one_letter(residue);
  if (aa < 0) return og_fail(OG_E_BADARG, std::string("not an amino-acid code: ") + residue);
  std::string err = og::append_residue(&c->s, *tpl, aa, or_default(phi, og::kDefaultPhi),
                                       or_default(psi, og::kDefaultPsi), or_default(omega, og::kDefaultOmega));
  if (!err.empty()) return og_fail(OG_E_DATA, err);
  c->dirty = true;
  return rebuild(c);
}

og_status og_chain_from_structure(int32_t n_residues, const char* residues, const char* chains,
                                  const int32_t* atoms_per_residue, const char* names, const int32_t* elements,
                                  const double* xyz, og_chain** out) {
  if (!out) return og_fail(OG_E_BADARG, "null argument");
  *out = nullptr;
  if (n_residues < 1 || !residues || !atoms_per_residue || !names || !xyz)
    return og_fail(OG_E_BADARG, "og_chain_from_structure: null array or no residues");
  auto c = std::make_unique<og_chain>();
  int64_t k = 0;
  for (int32_t r = 0; r < n_residues; ++r) {
    const int aa = og::aa_from_one_letter(residues[r]);
    if (aa < 0) return og_fail(OG_E_BADARG, std::string("not an amino-acid code: ") + residues[r]);
    if (atoms_per_residue[r] < 0) return og_fail(OG_E_BADARG, "negative atom count");
    og::PlacedResidue res;
    res.aa = aa;
    res.chain = chains ? chains[r] : 'A';
    for (int32_t a = 0; a < atoms_per_residue[r]; ++a, ++k) {
      og::PlacedAtom at;
      at.name.assign(names + 8 * k, strnlen(names + 8 * k, 8));
      if (elements) {
        if (elements[k] < 0 || elements[k] > 5) return og_fail(OG_E_BADARG, "element code out of range");
        at.element = static_cast<og::Element>(elements[k]);
      } else if (!og::element_from_symbol(at.name.substr(0, 1), &at.element)) {
        return og_fail(OG_E_DATA, "cannot determine the element of atom " + at.name);
      }
      at.pos = og::Vec3{xyz[3 * k], xyz[3 * k + 1], xyz[3 * k + 2]};
      res.atoms.push_back(at);
    }
    c->s.residues.push_back(std::move(res));
  }
  og_status st = rebuild(c.get());
  if (st != OG_OK) return st;
  *out = c.release();
  return OG_OK;
}

og_status og_chain_n_atoms(const og_chain* c, int32_t* n) {
  if (!c || !n) return og_fail(OG_E_BADARG, "null argument");
  *n = c->s.atom_count();
  return OG_OK;
}

og_status og_chain_n_residues(const og_chain* c, int32_t* n) {
  if (!c || !n) return og_fail(OG_E_BADARG, "null argument");
  *n = static_cast<int32_t>(c->s.residues.size());
  return OG_OK;
}

og_status og_chain_topology(og_chain* c, const og_topology** topo) {
  if (!c || !topo) return og_fail(OG_E_BADARG, "null argument");
  if (c->dirty) {
    og_status st = rebuild(c);
    if (st != OG_OK) return st;
  }
  *topo = &c->topo;
  return OG_OK;
}

og_status og_chain_get_positions(const og_chain* c, double* xyz) {
  if (!c || !xyz) return og_fail(OG_E_BADARG, "null argument");
  size_t k = 0;
  for (const auto& r : c->s.residues)
    for (const auto& a : r.atoms) {
      xyz[k++] = a.pos.x; xyz[k++] = a.pos.y; xyz[k++] = a.pos.z;
    }
  return OG_OK;
}

og_status og_chain_set_positions(og_chain* c, const double* xyz) {
  if (!c || !xyz) return og_fail(OG_E_BADARG, "null argument");
  size_t k = 0;
  for (auto& r : c->s.residues)
    for (auto& a : r.atoms) {
      a.pos.x = xyz[k++]; a.pos.y = xyz[k++]; a.pos.z = xyz[k++];
    }
  return OG_OK;
}

og_status og_chain_atom_info(const og_chain* c, int32_t atom, int32_t* residue, int32_t* atom_type, char name[8]) {
  if (!c) return og_fail(OG_E_BADARG, "null chain");
  int32_t k = 0;
  for (size_t r = 0; r < c->s.residues.size(); ++r)
    for (const auto& a : c->s.residues[r].atoms) {
      if (k == atom) {
        if (residue) *residue = static_cast<int32_t>(r);
        if (atom_type) *atom_type = og::classify(c->s.residues[r].aa, a.name);
        if (name) {
          std::strncpy(name, a.name.c_str(), 7);
          name[7] = '\0';
        }
        return OG_OK;
      }
      ++k;
    }
  return og_fail(OG_E_BADARG, "atom index out of range");
}

og_status og_chain_missing_params(const og_chain* c, int32_t* missing) {
  if (!c || !missing) return og_fail(OG_E_BADARG, "null argument");
  *missing = c->missing;
  return OG_OK;
}

void og_chain_free(og_chain* c) { delete c; }

}  // extern "C"
