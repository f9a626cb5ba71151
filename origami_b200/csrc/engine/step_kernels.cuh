// Element-wise and per-term kernels of one MD step: coordinate packing for
// the pair kernels, Born-radius finalisation, CHARMM bonded terms, the BAOAB
// sub-steps, SHAKE, replica exchange and per-system reductions.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ogk {

struct SysState {
  double temperature;   // K
  double kbt;           // kB T, kJ/mol
  double dof_corr;      // 3N / (3N - n_constraints) with SHAKE, else 1
  int32_t atom_begin;   // first padded atom
  int32_t n_atoms;      // real atoms
  int32_t status;       // kStatus* bits
  int32_t shake_flag;   // set by SHAKE clusters during one half step
  long long steps;      // completed steps
  long long shake_failures;
};

struct AtomArrays {
  int32_t n_padded;
  double* x; double* y; double* z;
  double* vx; double* vy; double* vz;
  double* rx; double* ry; double* rz;   // SHAKE reference positions
  unsigned long long* fx; unsigned long long* fy; unsigned long long* fz;
  unsigned long long* born_sum;
  const double* mass;
  const int32_t* atom_sys;    // -1 for padding
  const int32_t* local_idx;   // index within its system
  const double* q;
  const double* rho;          // intrinsic radius
  const double* rho_tilde;
  const double* srho;         // HCT scale * rho_tilde
  float* pq;                  // tile-SoA FP32 positions + charge
  float* gb;                  // tile-SoA R, 1/R, rho_tilde, s*rho_tilde
  double4* origin;            // per tile
  double* born_r;             // FP64 Born radii (force path)
  SysState* sys;
  int32_t* sys_nonfinite;     // per system, set by force kernels on NaN/Inf
};

// Packs FP64 positions into tile-relative FP32 coordinates, writes the tile
// origins, and (when zero_acc) clears the force and Born accumulators.
void launch_pack(const AtomArrays& a, bool zero_acc, cudaStream_t s);

// OBC-II map of the descreening integral to effective radii
// (energy/src/gb.rs:326-341), FP64.  The integral comes from integral_fp64
// when given, else from the fixed-point born_sum of the force path.  Radii go
// to out_r and, when write_gb, to the gb float4s the force pass reads.
// clamp_count (per system, optional) counts non-finite / non-positive
// inverse radii.
void launch_born_finalize(const AtomArrays& a, const double* integral_fp64, double* out_r, bool write_gb,
                          int32_t* clamp_count, cudaStream_t s);

// ------------------------------------------------------------------ bonded
struct BondedArgs {
  const double* x; const double* y; const double* z;
  int32_t n_bonds, n_angles, n_dihedrals, n_impropers;
  const int2* bond_atoms; const double* bond_k; const double* bond_r0;
  const int4* angle_atoms; const double* angle_k; const double* angle_t0;     // radians
  const int4* dih_atoms; const int2* dih_terms;                                 // [start, end)
  const double* term_k; const int32_t* term_n; const double* term_delta;      // radians
  const int4* imp_atoms; const double* imp_k; const double* imp_psi0;         // radians
  unsigned long long* fx; unsigned long long* fy; unsigned long long* fz;     // force mode
  double* energy;  // energy mode: one value per term (bonds, then angles, dihedrals, impropers)
  const int32_t* atom_sys;
  int32_t* sys_nonfinite;  // set when a term's force is NaN/Inf
};
void launch_bonded_forces(const BondedArgs& a, cudaStream_t s);
void launch_bonded_energies(const BondedArgs& a, cudaStream_t s);

// ------------------------------------------------------------------- BAOAB
struct StepArgs {
  AtomArrays at;
  double half_dt;
  double alpha;          // exp(-gamma dt)
  uint32_t seed_lo, seed_hi;
  int32_t use_shake;
};
// B (first half) + A (first half); stores SHAKE reference positions.
void launch_step_pre(const StepArgs& a, cudaStream_t s);
// [SHAKE velocity fix] + O + A (second half).
void launch_step_mid(const StepArgs& a, cudaStream_t s);
// [SHAKE velocity fix] + pack + zero accumulators.
void launch_step_post(const StepArgs& a, cudaStream_t s);
// B (second half), divergence check, step counter.
void launch_step_end(const StepArgs& a, cudaStream_t s);

struct ShakeArgs {
  double* x; double* y; double* z;
  const double* rx; const double* ry; const double* rz;
  const double* inv_mass;
  int32_t n_clusters;
  const int32_t* cluster_start;  // n_clusters + 1, into the constraint arrays
  const int32_t* cluster_sys;
  const int2* cons_atoms;
  const double* cons_d2;
  double tol_sq;
  int32_t max_iters;
  SysState* sys;
};
void launch_shake(const ShakeArgs& a, cudaStream_t s);

// Per-system deterministic sums of a per-atom (or per-term) array:
// out[s] = sum over [begin[s], end[s]) in a fixed order.
void launch_segment_sum(const double* v, const int32_t* begin, const int32_t* end, int32_t n_seg, double* out,
                        cudaStream_t s);

// Replica exchange (remd.rs:442-465): swap positions, forces and Born radii
// of two systems of equal size; velocities swap and are rescaled
// (system a receives b's velocities times scale_a and vice versa).
void launch_swap_systems(const AtomArrays& a, int32_t begin_a, int32_t begin_b, int32_t n, double scale_a,
                         double scale_b, cudaStream_t s);

// Soft cylindrical exit tunnel (cotranslate.rs:119-154 CylindricalTunnel):
// an atom whose projection on the axis (origin + t * direction, direction
// used as given -- a unit vector) lies within [0, length] and whose distance
// from the axis exceeds the radius feels k (d - radius) back toward the
// axis; added to the fixed-point forces of every real atom.
struct TunnelParams {
  double ox, oy, oz;  // axis origin, A
  double dx, dy, dz;  // axis direction
  double radius, length, k;  // A, A, kJ/mol/A^2
};
void launch_tunnel(const AtomArrays& a, const TunnelParams& t, cudaStream_t s);

// Kinetic energy per system: sum m v^2 / 2 / ACCEL (langevin.rs:469-475).
// Device-side replica exchange round (og_remd_run): per-system energies
// from the FP64 energy kernels' outputs, Metropolis on neighbouring
// temperature slots, temperature labels exchanged, velocities rescaled.
struct RemdArgs {
  SysState* sys;
  int32_t* sys_of_slot;   // n_slots: the system at each temperature slot
  const double* temps;    // n_slots ascending temperatures
  double* total;          // n_slots scratch: potential energy per system
  double* vscale;         // n_slots scratch: velocity factor per system
  long long* attempts;    // n_slots - 1 counters per slot pair
  long long* accepts;
  const double* e_lj; const double* e_coul; const double* e_gb; const double* e_self; const double* bonded_e;
  const int32_t* seg_begin;  // the engine's [atoms | bonds | angles | dihedrals | impropers] segments
  const int32_t* seg_end;
  int32_t n_slots;
  uint64_t seed;
};
void launch_remd_round(const AtomArrays& a, const RemdArgs& r, int parity, uint32_t round, cudaStream_t s);

void launch_kinetic(const AtomArrays& a, const int32_t* begin, const int32_t* end, int32_t n_sys, double* out,
                    cudaStream_t s);

}  // namespace ogk
