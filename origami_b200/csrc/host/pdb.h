// PDB output (io/src/pdb.rs): the record text of a chain laid out once,
// single-model files and multi-MODEL trajectories, and the trajectory
// handle behind the C ABI's og_trajectory (host frames, or engine frames
// copied to pinned memory asynchronously -- see og_trajectory_capture).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../../../include/origami_gpu.h"

namespace og {

// Everything of a chain's ATOM/TER records except the coordinates
// (io/src/pdb.rs:66-121): per atom the text of columns 1-30 and 55-78, the
// chain-boundary TER records written before an atom, and the closing TER.
struct PdbLayout {
  int n_atoms = 0;
  std::vector<std::string> head, tail;
  std::vector<std::string> ter_before;  // "" for none
  std::string final_ter;
};

PdbLayout pdb_layout(const og_chain* c);
void pdb_write_header(FILE* f, const char* title);
void pdb_write_atoms(FILE* f, const PdbLayout& l, const double* xyz);

}  // namespace og

struct og_trajectory {
  FILE* file = nullptr;
  og::PdbLayout layout;
  int64_t models = 0;  // MODEL blocks written
  // engine frames: two pinned host frames in flight, one device staging frame
  double* pinned[2] = {nullptr, nullptr};
  double* staging = nullptr;
  cudaEvent_t copied[2] = {nullptr, nullptr};
  int64_t pending[2] = {-1, -1};  // capture number held by each slot (-1 none)
  int64_t captures = 0;
};

// Writes the pending engine frames with capture numbers below `before`, in
// capture order (waiting for their copies); all of them by default, so that
// a host frame or END can follow.
og_status og_trajectory_flush(og_trajectory* t, int64_t before = INT64_MAX);
