// Host-side chemistry model: elements, amino acids, CHARMM36m atom typing,
// force-field parameter lookup, residue templates, the NeRF chain builder and
// the bonded topology graph.  This is the input side of the force engine: it
// turns a sequence into the flat per-atom / per-term arrays the CUDA kernels
// consume (see include/origami_gpu.h, og_topology).
//
// Every rule here restates origami's Rust host (paths relative to the
// reference's crates/ directory) so the arrays are identical to what origami
// would feed its own force code:
//   chem/src/element.rs, chem/src/amino_acid.rs, chem/src/atom_type.rs:164
//   chem/src/forcefield.rs:84-459, chem/src/topology_data.rs
//   geom/src/nerf.rs:15, geom/src/builder.rs:50-238
//   geom/src/topology_graph.rs:81-389
#pragma once

#include <array>
#include <cstdint>
#include <map>
#include <string>
#include <tuple>
#include <vector>

namespace og {

enum class Element : int8_t { H = 0, C = 1, N = 2, O = 3, P = 4, S = 5 };

double element_mass(Element e);      // chem/src/element.rs:27-37
double element_vdw(Element e);       // chem/src/element.rs:40-49 (Bondi)
char element_symbol(Element e);
bool element_from_symbol(const std::string& s, Element* out);

// AminoAcid::ALL order (chem/src/amino_acid.rs:31): the index doubles as the
// residue code in every array of this library.
constexpr int kNumAminoAcids = 20;
enum AminoAcid : int8_t {
  ALA, ARG, ASN, ASP, CYS, GLN, GLU, GLY, HIS, ILE,
  LEU, LYS, MET, PHE, PRO, SER, THR, TRP, TYR, VAL
};
int aa_from_one_letter(char c);                 // -1 when unknown
int aa_from_three_letter(const std::string& s); // -1 when unknown (case-insensitive)
const char* aa_three_letter(int aa);            // upper case, e.g. "ALA"
char aa_one_letter(int aa);

// CHARMM36 atom types in the declaration order of chem/src/atom_type.rs:18
// (that order is the Ord used to canonicalise parameter keys).
enum AtomType : int8_t {
  T_C, T_CA, T_CAI, T_CC, T_CT1, T_CT2, T_CT2A, T_CT3, T_CP1, T_CP2, T_CP3,
  T_CPH1, T_CPH2, T_CPT, T_CY,
  T_N, T_NH1, T_NH2, T_NH3, T_NC2, T_NR1, T_NR2, T_NY,
  T_O, T_OC, T_OH1,
  T_S,
  T_H, T_HA, T_HA1, T_HA2, T_HA3, T_HB1, T_HB2, T_HC, T_HP, T_HR1, T_HR3, T_HS,
  kNumAtomTypes
};
const char* atom_type_name(int t);
int atom_type_from_name(const std::string& s);  // -1 when not modelled
Element atom_type_element(int t);
// classify(aa, atom_name): chem/src/atom_type.rs:164.  -1 = not modelled.
int classify(int aa, const std::string& name);

// ---------------------------------------------------------------- force field
struct BondParams { double k, r0; };               // kcal/mol/A^2, A
struct AngleParams { double k, theta0_deg; };       // kcal/mol/rad^2, deg
struct DihedralTerm { double k; int n; double delta_deg; };
struct ImproperParams { double k, psi0_deg; };
struct NonbondedParams {
  double epsilon, rmin_half;          // epsilon positive (kcal/mol)
  bool has14;
  double epsilon_14, rmin_half_14;
};

class ForceField {
 public:
  // Loads the table written by origami_b200/data/make_tables.py.  Returns an
  // empty string on success, else a message.
  std::string load(const std::string& path);
  const BondParams* bond(int a, int b) const;
  const AngleParams* angle(int a, int b, int c) const;
  const std::vector<DihedralTerm>* dihedral(int a, int b, int c, int d) const;
  const ImproperParams* improper(int a, int b, int c, int d) const;
  const NonbondedParams* nonbonded(int t) const;
  bool partial_charge(int aa, const std::string& name, double* q) const;

 private:
  using K2 = std::pair<int, int>;
  using K3 = std::tuple<int, int, int>;
  using K4 = std::tuple<int, int, int, int>;
  std::map<K2, BondParams> bonds_;
  std::map<K3, AngleParams> angles_;
  std::map<K4, std::vector<DihedralTerm>> dihedrals_;
  std::map<K2, std::vector<DihedralTerm>> wildcard_dihedrals_;
  std::map<K4, ImproperParams> impropers_;
  std::map<K2, ImproperParams> wildcard_impropers_;
  std::map<int, NonbondedParams> nonbonded_;
  std::map<std::pair<int, std::string>, double> charges_;
};

// ---------------------------------------------------------- residue templates
struct TemplateAtom {
  std::string name;
  Element element;
  std::string bond_to, angle_at, dihedral_to;
  double bond_length, bond_angle;
  char kind;      // 'F' fixed dihedral, 'C' chi_n, 'P' chi_n + value
  int chi_n;
  double value;
};
struct ResidueTemplate {
  bool has_amide_h = true;
  bool is_glycine = false;
  std::vector<double> default_chi;
  std::vector<TemplateAtom> sidechain;
};
class Templates {
 public:
  std::string load(const std::string& path);
  const ResidueTemplate& get(int aa) const { return res_[aa]; }
 private:
  std::array<ResidueTemplate, kNumAminoAcids> res_;
};

// ------------------------------------------------------------------ structure
struct Vec3 { double x, y, z; };
struct PlacedAtom { std::string name; Element element; Vec3 pos; };
struct PlacedResidue { int aa; char chain; std::vector<PlacedAtom> atoms; };
struct Structure {
  std::vector<PlacedResidue> residues;
  int atom_count() const;
};

Vec3 place_atom(Vec3 a, Vec3 b, Vec3 c, double length, double angle, double dihedral);

// Default extended-chain torsions (geom/src/builder.rs:20-22).
extern const double kDefaultPhi, kDefaultPsi, kDefaultOmega;
// Appends one residue with NeRF (geom/src/builder.rs:78 append_residue).
std::string append_residue(Structure* s, const Templates& tpl, int aa, double phi,
                           double psi, double omega);

// ----------------------------------------------------------------- topology
struct Topology {
  std::vector<std::array<int, 2>> bonds;       // a < b, sorted
  std::vector<std::array<int, 3>> angles;      // (a, central, c)
  std::vector<std::array<int, 4>> dihedrals;   // canonical b < c
  std::vector<std::array<int, 4>> impropers;   // central first
  std::vector<std::vector<int>> bonded_to;     // sorted adjacency
};
Topology build_topology(const Structure& s, const Templates& tpl);

// Per-pair classification of geom/src/topology_graph.rs:81-112 as graph
// distance: 1-2 and 1-3 pairs are excluded, 1-4 pairs are flagged.
struct ExclusionPair { int i, j; int8_t kind; };  // kind 1 = excluded, 2 = 1-4
std::vector<ExclusionPair> build_exclusions(const Topology& t, int n_atoms);

}  // namespace og
