// The og_chain behind the C ABI's opaque handle: the placed structure
// (residues, atom names, elements, positions) plus the flat arrays that back
// its og_topology.  Shared by the chain and PDB translation units.
#pragma once

#include <cstdint>
#include <vector>

#include "../../../include/origami_gpu.h"
#include "model.h"

struct og_chain {
  og::Structure s;
  // Flattened arrays backing `topo`.
  std::vector<double> charge, rmin, eps, rmin14, eps14, rho, scale, mass;
  std::vector<int32_t> element, atom_type, residue_of;
  std::vector<int32_t> bond_atoms, angle_atoms, dih_atoms, dih_start, term_n, imp_atoms;
  std::vector<double> bond_k, bond_r0, angle_k, angle_t0, term_k, term_delta, imp_k, imp_psi0;
  std::vector<int32_t> excl_atoms, cons_atoms;
  std::vector<int8_t> excl_kind;
  std::vector<double> cons_d;
  int32_t missing = 0;
  og_topology topo{};
  bool dirty = true;
};
