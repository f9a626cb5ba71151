// Analytical PowerSasa surface term on the GPU: per-atom accessible area
// (spherical Gauss-Bonnet over the exposed boundary arcs) and its exact
// analytical gradient, restating crates/energy/src/powersasa/ (see sasa.cu
// for the per-function citations).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "step_kernels.cuh"

namespace ogk {

// Per-atom capacities of the on-chip boundary arrangement.  An atom that
// exceeds one marks its system with kStatusSasaOverflow (the host reports
// OG_E_UNSUPPORTED) instead of producing a wrong force.  Protein atoms reach
// about 90 caps, 46 of them left after contained caps are dropped, 72
// transitions on one circle and 19 exposed arcs.
// Arrangement capacities per atom: the default kernels' (four warps per
// block, five blocks per SM) and the large ones for the atoms that exceed
// them (caps cutting the atom's sphere, transitions of one batch of circles,
// exposed arcs).
constexpr int kSasaMaxCaps = 112;
constexpr int kSasaMaxTrans = 96;
constexpr int kSasaMaxArcs = 36;
constexpr int kSasaBigCaps = 254;
constexpr int kSasaBigTrans = 254;
constexpr int kSasaBigArcs = 128;
constexpr int kStatusSasaOverflow = 8;

// Probes of the accessible-component count (arrangement.rs:327-391).
constexpr int kSasaProbes = 500;

// One Gauss-Bonnet term of some atom i's boundary, as the force kernel's
// second stage differentiates it: an arc of cap k (owner atom k) whose start
// and end vertices are shared with the caps of atoms l and m (roots ss, se;
// vertexed = 0 for a full circle or an unlinked vertex), or a vertex where
// the boundary passes from the cap of atom k to that of atom l.
struct SasaArcTerm {
  int32_t i, k, l, m;
  double theta;
  int32_t ss, se, vertexed, pad;
};
struct SasaVertexTerm {
  int32_t i, k, l, sign;
};

struct SasaArgs {
  const double* x;
  const double* y;
  const double* z;
  const double* radius;       // per padded atom: vdW + 1.4 A probe
  const double* gamma;        // per padded atom: surface tension, kJ/mol/A^2
  const int32_t* tasks;       // padded atom indices to evaluate
  int32_t n_tasks;
  const int32_t* atom_sys;    // -1 for padding
  const int2* sys_tiles;      // per system: (first tile, tile count)
  const double4* origin;      // per tile: centroid, w = bounding radius
  double r_max;               // largest SASA radius of any atom
  unsigned long long* fx;     // fixed-point forces (kForceScale)
  unsigned long long* fy;
  unsigned long long* fz;
  double* area;               // per padded atom (area kernels)
  double* energy;             // per padded atom gamma * area (area kernels)
  const double* probes;       // kSasaProbes x 3 unit vectors
  const int32_t* probe_adj_begin;  // CSR adjacency of the probe graph
  const int16_t* probe_adj;
  SysState* sys;
  // force path: term records of every atom's boundary, appended through
  // counts[0] (arcs) and counts[1] (vertices), capacity `term_cap` each;
  // counts[2] counts the atoms queued in overflow[] (capacity overflow_cap)
  // for the large-capacity kernels; counts[3] is the next atom of the
  // default-capacity kernels' work queue
  SasaArcTerm* arc_terms;
  SasaVertexTerm* vertex_terms;
  int32_t* counts;
  int32_t term_cap;
  int32_t* overflow;
  int32_t overflow_cap;
};

// F_x += gamma_i R_i^2 (sum_arcs [theta dcos + cos_alpha dtheta] + sum_vertices
// d epsilon) over every task atom i with a bounded boundary: a boundary
// kernel (one warp per atom) appends term records, a second kernel
// differentiates one record per thread.  counts must be zero on entry (the
// launcher clears them on the stream).
void launch_sasa_forces(const SasaArgs& a, cudaStream_t s);

// area[i] and energy[i] = gamma_i area[i] for every task atom i (0 buried,
// 4 pi R^2 exposed).
void launch_sasa_areas(const SasaArgs& a, cudaStream_t s);

// Shrake-Rupley area (crates/energy/src/sasa.rs:65-110) with n_dots
// Fibonacci test points per task atom; same outputs as launch_sasa_areas.
void launch_shrake_rupley(const SasaArgs& a, const double* dots, int n_dots, cudaStream_t s);

// Sets the kernels' shared-memory limits; call once before the first launch
// (outside stream capture).
cudaError_t sasa_prepare();

}  // namespace ogk
