// Device helpers shared by the engine's kernels: fixed-point accumulation,
// the counter-based noise generator, mbarrier + bulk-copy (TMA) primitives
// with bounded waits, and the physical constants of origami's force field.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ogk {

// ------------------------------------------------------------- constants
// origami's constants (crates/energy/src/units.rs:4, nonbonded.rs:34,
// gb.rs:20-40, dynamics/src/langevin.rs:44-47).
constexpr double kKcalToKj = 4.184;
constexpr double kCoulomb = 332.0637;
constexpr double kEpsWater = 78.5;
constexpr double kObcAlpha = 1.0, kObcBeta = 0.8, kObcGamma = 4.85;
constexpr double kObcOffset = 0.09;
constexpr double kBoltzmann = 8.314462618e-3;
constexpr double kAccel = 1.0e-4;

// Fixed-point scales.  Forces: 2^32 units per kJ/mol/A (|F| < 2^31 kJ/mol/A).
// Born descreening integral: 2^40 units per 1/A.
constexpr double kForceScale = 4294967296.0;
constexpr double kForceUnscale = 1.0 / 4294967296.0;
constexpr double kBornScale = 1099511627776.0;
constexpr double kBornUnscale = 1.0 / 1099511627776.0;

// Tile geometry: 32 atoms per tile (one warp lane per atom).
constexpr int kTile = 32;

// Tile-SoA layout of the FP32 per-atom arrays the pair kernels stream: tile
// t occupies 128 consecutive floats, four 32-float columns c = 0..3, so one
// 512-byte bulk copy moves a whole tile and a 16-byte shared-memory load
// yields one column for four consecutive atoms.
__host__ __device__ __forceinline__ int soa_index(int atom, int col) {
  return ((atom >> 5) << 7) + (col << 5) + (atom & 31);
}

// Status bits of a system (og_system_stats / og_step).
constexpr int kStatusDiverged = 1;
constexpr int kStatusShakeFail = 2;
constexpr int kStatusTimeout = 4;

__device__ __forceinline__ void add_fixed(unsigned long long* p, double v, double scale) {
  long long q = __double2ll_rn(v * scale);
  atomicAdd(p, static_cast<unsigned long long>(q));
}

// ----------------------------------------------------------- noise (O step)
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11).  Counter = (atom,
// step_lo, step_hi, system), key = (seed_lo, seed_hi).  Four 32-bit outputs
// feed two Box-Muller pairs; the first three normals are the x, y, z noise
// of one atom in one step.  The oracle restates the same generator.
struct U4 { uint32_t x, y, z, w; };

__host__ __device__ __forceinline__ void mulhilo(uint32_t a, uint32_t b, uint32_t* hi, uint32_t* lo) {
  uint64_t p = static_cast<uint64_t>(a) * b;
  *hi = static_cast<uint32_t>(p >> 32);
  *lo = static_cast<uint32_t>(p);
}

__host__ __device__ __forceinline__ U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
  for (int r = 0; r < 10; ++r) {
    uint32_t hi0, lo0, hi1, lo1;
    mulhilo(0xD2511F53u, c.x, &hi0, &lo0);
    mulhilo(0xCD9E8D57u, c.z, &hi1, &lo1);
    U4 n{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
    c = n;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}

// Uniform in (0, 1] from 32 bits (never 0, so log() is finite).
__host__ __device__ __forceinline__ double u32_to_open01(uint32_t v) {
  return (static_cast<double>(v) + 1.0) * (1.0 / 4294967296.0);
}

// ---------------------------------------------------- mbarrier / bulk copy
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n"
      " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}

// Bounded wait: returns false after `limit` polls (the caller records a
// timeout and stops using the buffer).  try_wait itself suspends for a
// hardware time slice, so the limit corresponds to well over a second.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t phase, uint32_t limit = 1u << 22) {
  for (uint32_t it = 0; it < limit; ++it)
    if (mbar_try_wait(bar, phase)) return true;
  return false;
}

// One-dimensional TMA bulk copy global -> shared, completion counted on an
// mbarrier.  Both addresses 16-byte aligned, size a multiple of 16 bytes.
__device__ __forceinline__ void bulk_g2s(void* smem_dst, const void* gmem_src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(smem_dst)),
      "l"(gmem_src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// ------------------------------------------------------------- reductions
__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

}  // namespace ogk
