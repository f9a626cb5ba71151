// Elements, amino acids and CHARMM36 atom typing.
// classify() restates chem/src/atom_type.rs:164-486 rule for rule.
#include <cctype>
#include <cstring>

#include "model.h"

namespace og {

double element_mass(Element e) {
  switch (e) {
    case Element::H: return 1.008;
    case Element::C: return 12.011;
    case Element::N: return 14.007;
    case Element::O: return 15.999;
    case Element::P: return 30.974;
    case Element::S: return 32.06;
  }
  return 0.0;
}

double element_vdw(Element e) {
  switch (e) {
    case Element::H: return 1.20;
    case Element::C: return 1.70;
    case Element::N: return 1.55;
    case Element::O: return 1.52;
    case Element::P: return 1.80;
    case Element::S: return 1.80;
  }
  return 0.0;
}

char element_symbol(Element e) { return "HCNOPS"[static_cast<int>(e)]; }

bool element_from_symbol(const std::string& s, Element* out) {
  if (s.size() != 1) return false;
  const char* p = std::strchr("HCNOPS", s[0]);
  if (!p || !*p) return false;
  *out = static_cast<Element>(p - "HCNOPS");
  return true;
}

static const char* kAA3[kNumAminoAcids] = {
    "ALA", "ARG", "ASN", "ASP", "CYS", "GLN", "GLU", "GLY", "HIS", "ILE",
    "LEU", "LYS", "MET", "PHE", "PRO", "SER", "THR", "TRP", "TYR", "VAL"};
static const char kAA1[kNumAminoAcids + 1] = "ARNDCQEGHILKMFPSTWYV";

int aa_from_one_letter(char c) {
  c = static_cast<char>(std::toupper(static_cast<unsigned char>(c)));
  for (int i = 0; i < kNumAminoAcids; ++i)
    if (kAA1[i] == c) return i;
  return -1;
}

int aa_from_three_letter(const std::string& s) {
  if (s.size() != 3) return -1;
  std::string u = s;
  for (auto& ch : u) ch = static_cast<char>(std::toupper(static_cast<unsigned char>(ch)));
  for (int i = 0; i < kNumAminoAcids; ++i)
    if (u == kAA3[i]) return i;
  return -1;
}

const char* aa_three_letter(int aa) { return (aa >= 0 && aa < kNumAminoAcids) ? kAA3[aa] : "UNK"; }
char aa_one_letter(int aa) { return (aa >= 0 && aa < kNumAminoAcids) ? kAA1[aa] : 'X'; }

static const char* kTypeNames[kNumAtomTypes] = {
    "C", "CA", "CAI", "CC", "CT1", "CT2", "CT2A", "CT3", "CP1", "CP2", "CP3",
    "CPH1", "CPH2", "CPT", "CY",
    "N", "NH1", "NH2", "NH3", "NC2", "NR1", "NR2", "NY",
    "O", "OC", "OH1",
    "S",
    "H", "HA", "HA1", "HA2", "HA3", "HB1", "HB2", "HC", "HP", "HR1", "HR3", "HS"};

const char* atom_type_name(int t) { return (t >= 0 && t < kNumAtomTypes) ? kTypeNames[t] : "?"; }

int atom_type_from_name(const std::string& s) {
  for (int i = 0; i < kNumAtomTypes; ++i)
    if (s == kTypeNames[i]) return i;
  return -1;
}

Element atom_type_element(int t) {
  if (t <= T_CY) return Element::C;
  if (t <= T_NY) return Element::N;
  if (t <= T_OH1) return Element::O;
  if (t == T_S) return Element::S;
  return Element::H;
}

namespace {
bool any_of(const std::string& n, std::initializer_list<const char*> names) {
  for (const char* x : names)
    if (n == x) return true;
  return false;
}
}  // namespace

int classify(int aa, const std::string& n) {
  // Backbone, uniform except Pro and Gly.
  if (aa == PRO) {
    if (n == "N") return T_N;
    if (n == "CA") return T_CP1;
    if (n == "C") return T_C;
    if (n == "O") return T_O;
    if (n == "HA") return T_HB1;
  } else if (aa == GLY) {
    if (n == "N") return T_NH1;
    if (n == "CA") return T_CT2;
    if (n == "C") return T_C;
    if (n == "O") return T_O;
    if (n == "H") return T_H;
    if (n == "HA2" || n == "HA3") return T_HB2;
  }
  if (n == "N") return T_NH1;
  if (n == "CA") return T_CT1;
  if (n == "C") return T_C;
  if (n == "O") return T_O;
  if (n == "H") return T_H;
  if (n == "HA") return T_HB1;

  switch (aa) {
    case GLY: return -1;
    case ALA:
      if (n == "CB") return T_CT3;
      if (any_of(n, {"HB1", "HB2", "HB3"})) return T_HA3;
      return -1;
    case VAL:
      if (n == "CB") return T_CT1;
      if (n == "HB") return T_HA1;
      if (any_of(n, {"CG1", "CG2"})) return T_CT3;
      if (any_of(n, {"HG11", "HG12", "HG13", "HG21", "HG22", "HG23"})) return T_HA3;
      return -1;
    case LEU:
      if (n == "CB") return T_CT2;
      if (any_of(n, {"HB2", "HB3"})) return T_HA2;
      if (n == "CG") return T_CT1;
      if (n == "HG") return T_HA1;
      if (any_of(n, {"CD1", "CD2"})) return T_CT3;
      if (any_of(n, {"HD11", "HD12", "HD13", "HD21", "HD22", "HD23"})) return T_HA3;
      return -1;
    case ILE:
      if (n == "CB") return T_CT1;
      if (n == "HB") return T_HA1;
      if (n == "CG2") return T_CT3;
      if (any_of(n, {"HG21", "HG22", "HG23"})) return T_HA3;
      if (n == "CG1") return T_CT2;
      if (any_of(n, {"HG12", "HG13"})) return T_HA2;
      if (n == "CD1") return T_CT3;
      if (any_of(n, {"HD11", "HD12", "HD13"})) return T_HA3;
      return -1;
    case MET:
      if (any_of(n, {"CB", "CG"})) return T_CT2;
      if (any_of(n, {"HB2", "HB3", "HG2", "HG3"})) return T_HA2;
      if (n == "SD") return T_S;
      if (n == "CE") return T_CT3;
      if (any_of(n, {"HE1", "HE2", "HE3"})) return T_HA3;
      return -1;
    case PRO:
      if (any_of(n, {"CB", "CG"})) return T_CP2;
      if (n == "CD") return T_CP3;
      if (any_of(n, {"HB2", "HB3", "HG2", "HG3", "HD2", "HD3"})) return T_HA2;
      return -1;
    case SER:
      if (n == "CB") return T_CT2;
      if (any_of(n, {"HB2", "HB3"})) return T_HA2;
      if (n == "OG") return T_OH1;
      if (n == "HG") return T_H;
      return -1;
    case THR:
      if (n == "CB") return T_CT1;
      if (n == "HB") return T_HA1;
      if (n == "OG1") return T_OH1;
      if (n == "HG1") return T_H;
      if (n == "CG2") return T_CT3;
      if (any_of(n, {"HG21", "HG22", "HG23"})) return T_HA3;
      return -1;
    case CYS:
      if (n == "CB") return T_CT2;
      if (any_of(n, {"HB2", "HB3"})) return T_HA2;
      if (n == "SG") return T_S;
      if (n == "HG") return T_HS;
      return -1;
    case ASN:
      if (n == "CB") return T_CT2;
      if (any_of(n, {"HB2", "HB3"})) return T_HA2;
      if (n == "CG") return T_CC;
      if (n == "OD1") return T_O;
      if (n == "ND2") return T_NH2;
      if (any_of(n, {"HD21", "HD22"})) return T_H;
      return -1;
    case GLN:
      if (n == "CB") return T_CT2;
      if (any_of(n, {"HB2", "HB3"})) return T_HA2;
      if (n == "CG") return T_CT2;
      if (any_of(n, {"HG2", "HG3"})) return T_HA2;
      if (n == "CD") return T_CC;
      if (n == "OE1") return T_O;
      if (n == "NE2") return T_NH2;
      if (any_of(n, {"HE21", "HE22"})) return T_H;
      return -1;
    case ASP:
      if (n == "CB") return T_CT2A;
      if (any_of(n, {"HB2", "HB3"})) return T_HA2;
      if (n == "CG") return T_CC;
      if (any_of(n, {"OD1", "OD2"})) return T_OC;
      return -1;
    case GLU:
      if (n == "CB") return T_CT2A;
      if (any_of(n, {"HB2", "HB3"})) return T_HA2;
      if (n == "CG") return T_CT2;
      if (any_of(n, {"HG2", "HG3"})) return T_HA2;
      if (n == "CD") return T_CC;
      if (any_of(n, {"OE1", "OE2"})) return T_OC;
      return -1;
    case LYS:
      if (any_of(n, {"CB", "CG", "CD", "CE"})) return T_CT2;
      if (any_of(n, {"HB2", "HB3", "HG2", "HG3", "HD2", "HD3", "HE2", "HE3"})) return T_HA2;
      if (n == "NZ") return T_NH3;
      if (any_of(n, {"HZ1", "HZ2", "HZ3"})) return T_HC;
      return -1;
    case ARG:
      if (any_of(n, {"CB", "CG", "CD"})) return T_CT2;
      if (any_of(n, {"HB2", "HB3", "HG2", "HG3", "HD2", "HD3"})) return T_HA2;
      if (n == "NE") return T_NC2;
      if (n == "HE") return T_HC;
      if (n == "CZ") return T_C;
      if (any_of(n, {"NH1", "NH2"})) return T_NC2;
      if (any_of(n, {"HH11", "HH12", "HH21", "HH22"})) return T_HC;
      return -1;
    case HIS:
      if (n == "CB") return T_CT2;
      if (any_of(n, {"HB2", "HB3"})) return T_HA2;
      if (n == "CG") return T_CPH1;
      if (n == "ND1") return T_NR1;
      if (n == "HD1") return T_H;
      if (n == "CE1") return T_CPH2;
      if (n == "HE1") return T_HR1;
      if (n == "NE2") return T_NR2;
      if (n == "CD2") return T_CPH1;
      if (n == "HD2") return T_HR3;
      return -1;
    case PHE:
      if (n == "CB") return T_CT2;
      if (any_of(n, {"HB2", "HB3"})) return T_HA2;
      if (any_of(n, {"CG", "CD1", "CD2", "CE1", "CE2", "CZ"})) return T_CA;
      if (any_of(n, {"HD1", "HD2", "HE1", "HE2", "HZ"})) return T_HP;
      return -1;
    case TYR:
      if (n == "CB") return T_CT2;
      if (any_of(n, {"HB2", "HB3"})) return T_HA2;
      if (any_of(n, {"CG", "CD1", "CD2", "CE1", "CE2", "CZ"})) return T_CA;
      if (any_of(n, {"HD1", "HD2", "HE1", "HE2"})) return T_HP;
      if (n == "OH") return T_OH1;
      if (n == "HH") return T_H;
      return -1;
    case TRP:
      if (n == "CB") return T_CT2;
      if (any_of(n, {"HB2", "HB3"})) return T_HA2;
      if (n == "CG") return T_CY;
      if (n == "CD1") return T_CA;
      if (n == "HD1") return T_HP;
      if (n == "NE1") return T_NY;
      if (n == "HE1") return T_H;
      if (n == "CE2") return T_CPT;
      if (n == "CD2") return T_CPT;
      if (any_of(n, {"CE3", "CZ2"})) return T_CAI;
      if (any_of(n, {"CZ3", "CH2"})) return T_CA;
      if (any_of(n, {"HE3", "HZ2", "HZ3", "HH2"})) return T_HP;
      return -1;
    default:
      return -1;
  }
}

}  // namespace og
