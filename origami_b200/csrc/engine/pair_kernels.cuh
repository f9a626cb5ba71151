// Tiled all-pairs / tile-list pair kernels (FP32 pair math, FP64 per-tile
// accumulation, 64-bit fixed-point results) and the FP64 energy kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ogk {

// One unit of pair work: `n_i_tiles` (<= warps per CTA) consecutive i-tiles of
// one system against the j-tiles jlist[j_begin, j_end).
struct PairWork {
  int32_t i_tile0;
  int32_t n_i_tiles;
  int32_t j_begin;
  int32_t j_end;
};

// Exclusion masks of one ordered (i-tile, j-tile) pair: for i-lane l, bit k
// of ex[l] marks pair (i0+l, j0+k) as excluded (1-2, 1-3 or self), bit k of
// m14[l] as a 1-4 pair.  Entries of one i-tile are sorted by j-tile.
struct TileMaskRef {
  int32_t j_tile;
  int32_t offset;  // index of the 32-word block in the mask arrays
};

struct PairArgs {
  // per padded atom
  // FP32 per-atom data in tile-SoA layout (see soa_index in common.cuh):
  const float* pq;    // columns x_rel, y_rel, z_rel (A, from the tile origin), charge (e)
  const float* lj;    // columns rmin_half, sqrt(eps), rmin_half_14, sqrt(eps_14)   (kcal/mol)
  const float* gb;    // columns R_born, 1/R_born, rho_tilde, s*rho_tilde
  const double4* origin;  // per tile
  const int32_t* atom_valid;  // 1 for real atoms
  // work
  const PairWork* work;
  int32_t n_work;
  const int32_t* jlist;
  // cutoff mode: per i-block first tile, the end of its culled j range in
  // jlist (the work items' j_end is clamped to it); NULL for all pairs
  const int32_t* seg_end;
  const int32_t* mask_begin;  // per tile: first TileMaskRef, mask_begin[t+1] = end
  const TileMaskRef* mask_refs;
  const uint32_t* mask_ex;
  const uint32_t* mask_14;
  // outputs (fixed point)
  unsigned long long* fx;
  unsigned long long* fy;
  unsigned long long* fz;
  unsigned long long* born_sum;
  // cutoffs squared (INFINITY = none) and constants
  float nb_c2, gb_c2, born_c2;
  float inv_rc3;     // 1/Rc^3 of the reaction field (0 without cutoff)
  float coul_kj;     // 332.0637 * 4.184
  float lj_kj12;     // 12 * 4.184
  float gb_pref_kj;  // (1 - 1/78.5) * 332.0637 * 4.184
  int32_t* error_flag;
  // persistent launches: the work-queue head (zeroed before each launch)
  int32_t* queue;
  // per-system "a force or Born sum was NaN/Inf" flags (fixed point cannot
  // carry a NaN, so it is recorded here and turned into divergence)
  const int32_t* atom_sys;
  int32_t* sys_nonfinite;
  // Near-field tiles (those carrying exclusion / 1-4 masks: the bonded
  // neighbourhood, where large pair forces cancel against the bonded terms)
  // are evaluated in FP64 from these arrays.
  const double* x64; const double* y64; const double* z64;
  const double* q64;
  const double* rmin64; const double* eps64; const double* rmin14_64; const double* eps14_64;
  const double* born_r64;
  double nb_c2_64, gb_c2_64, inv_rc3_64;
};

// One i-block of a pair work list: W i-tiles from i_tile0 against the j-tiles
// jlist[jb, je).
struct CutBlock {
  int32_t i_tile0, n_i_tiles, jb, je;
};
// Cutoff-mode j lists, rebuilt from the tile origins every force evaluation:
// for each i-block, the j-tiles of jlist_all[jb, je) whose bounding sphere
// comes within `cutoff` of any of the block's tile spheres, kept in order and
// compacted to the front of the same range of jlist_out; seg_end[i_tile0]
// receives the new end.  No atom pair within the cutoff is dropped (sphere
// bounds, FP64, 1e-3 A margin); the pair kernels still apply the cutoff per
// pair.
void launch_cut_lists(const CutBlock* blocks, int32_t n_blocks, const int32_t* jlist_all, const double4* origin,
                      double cutoff, int32_t* jlist_out, int32_t* seg_end, cudaStream_t s);

// How a pair pass is launched.  shape: 0 = 8 i-tiles per CTA (256 atoms)
// at the default occupancy target (Born 4 CTAs/SM, force 2), 1 = 4 i-tiles
// per CTA (128 atoms) at twice the CTAs, 2 = 8 i-tiles at 3 CTAs/SM; force
// pass only: 3 = two i-tiles per warp (k_force_ip), 8 warps, 16 i-tiles per
// CTA at 2 CTAs/SM, 4 = the same with 4 warps (8 i-tiles) at 4 CTAs/SM, 5 =
// 4 warps at 5 CTAs/SM (96 registers), 6 = at 6 CTAs/SM (80 registers);
// persistent: resident CTAs taking items from PairArgs::queue instead of
// one CTA per item.  The work list must be built for
// pair_shape_tiles(shape) i-tiles per item.
struct PairLaunch {
  int shape = 0;
  bool persistent = false;
};
int pair_shape_tiles(int shape);
constexpr int kBornShapes = 3;   // shapes 0..2
constexpr int kForceShapes = 7;  // shapes 0..6

void launch_born_pass(const PairArgs& a, const PairLaunch& c, cudaStream_t s);
// Far field (tiles without exclusion masks), FP32.
void launch_force_pass(const PairArgs& a, const PairLaunch& c, cudaStream_t s);
// Near field: near[k] = (i_tile, j_tile, mask block of (i_tile, j_tile), 0)
// for every unordered tile pair (i_tile <= j_tile) that carries masks, FP64;
// each pair once, both atoms' forces.
void launch_near_force64(const PairArgs& a, const int4* near, int n_near, cudaStream_t s);

// FP64 energy evaluation, one thread per i atom over every j of its system.
struct EnergyArgs {
  const double* x; const double* y; const double* z;
  const double* q;
  const double* rmin; const double* eps; const double* rmin14; const double* eps14;
  const double* rho_tilde; const double* srho;  // srho = scale * rho_tilde
  const double* born_r;                          // FP64 Born radii (output of born64)
  const int32_t* atom_sys;
  const int32_t* sys_begin;  // per system: first padded atom
  const int32_t* sys_count;  // real atoms
  const int32_t* excl_row;   // CSR over padded atoms: exclusion partners (both directions)
  const int32_t* excl_col;
  const int8_t* excl_kind;
  int32_t n_atoms_padded;
  double nb_c2;    // INFINITY = all pairs
  double born_c2;
  double kappa, crf;  // reaction field constants (0 without cutoff)
  // outputs, per padded atom
  double* integral;   // born64
  double* e_lj; double* e_coul; double* e_gb; double* e_self; int32_t* n_pairs;
  // Each i atom's partners are split into n_chunks j ranges, one thread
  // each (so that a single chain fills the GPU); with more than one, the
  // range sums go to part ([3][n_chunks][n_atoms_padded] doubles: Born
  // integral or LJ, Coulomb, GB) and part_pairs, and are added in range
  // order by a second kernel.
  int32_t n_chunks;
  double* part;
  int32_t* part_pairs;
};

void launch_born64(const EnergyArgs& a, cudaStream_t s);
void launch_energy64(const EnergyArgs& a, cudaStream_t s);
// j ranges per i atom for the FP64 energy path: enough threads for eight
// 128-thread blocks per SM, at least 64 partners per range, at most 32.
int energy_chunks(int n_atoms_padded, int max_system_atoms, int n_sm);

}  // namespace ogk
