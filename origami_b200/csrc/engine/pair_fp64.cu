// FP64 pair kernels: the near-field force tiles of the force path and the
// energy path (Born radii and LJ / Coulomb / GB pair energies).
#include <algorithm>
#include <cmath>

#include "common.cuh"
#include "pair_kernels.cuh"

namespace ogk {

// ------------------------------------------------------- FP64 near field
// One warp per unordered near-field tile pair (i-tile <= j-tile) -- the
// tiles that carry exclusion / 1-4 masks, i.e. the bonded neighbourhood
// where the large LJ and Coulomb pair forces cancel against the bonded terms.
// FP64 throughout, the terms of forces_nonbonded.rs:196-232 +
// forces_gb.rs:82-111 with their square roots and divisions rewritten as
// reciprocal square roots and products (equal up to rounding; see the pair
// loop).  Each pair is evaluated once (Newton's third law):
// the j-tile's atoms are staged in the warp's shared memory, lane l meets
// partner (l + k) mod 32 at step k, so within a step every lane touches a
// different partner and the j-side sums need no atomics.  On a diagonal tile
// pair steps 1..16 cover every pair once (step 16 on the lower half-warp
// only).  The pair coefficient is symmetric in i and j, so the j-side force
// is exactly the negated i-side term.
namespace {

constexpr int kNearWarps = 4;

// The j-tile staged per warp: eps as its square root (the LJ mixing rule
// sqrt(eps_i eps_j) as a product) and the Born radius with its inverse.
struct NearTile {
  double x[kTile], y[kTile], z[kTile], q[kTile], r[kTile], ir[kTile];
  double rmin[kTile], seps[kTile], rmin14[kTile], seps14[kTile];
  double fx[kTile], fy[kTile], fz[kTile];
  int32_t valid[kTile];
};

__global__ void __launch_bounds__(kNearWarps * 32) k_near64(PairArgs a, const int4* __restrict__ near, int n_near) {
  __shared__ NearTile tiles[kNearWarps];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wid = blockIdx.x * kNearWarps + warp;
  if (wid >= n_near) return;
  NearTile& t = tiles[warp];
  const int4 w = near[wid];  // i_tile, j_tile (>= i_tile), mask block of (i_tile, j_tile)
  const int i = w.x * kTile + lane;
  const int jl = w.y * kTile + lane;  // this lane's j atom, staged for the warp
  t.x[lane] = a.x64[jl];
  t.y[lane] = a.y64[jl];
  t.z[lane] = a.z64[jl];
  t.q[lane] = a.q64[jl];
  t.r[lane] = a.born_r64[jl];
  t.ir[lane] = 1.0 / a.born_r64[jl];
  t.rmin[lane] = a.rmin64[jl];
  t.seps[lane] = sqrt(a.eps64[jl]);
  t.rmin14[lane] = a.rmin14_64[jl];
  t.seps14[lane] = sqrt(a.eps14_64[jl]);
  t.valid[lane] = a.atom_valid[jl];
  t.fx[lane] = t.fy[lane] = t.fz[lane] = 0.0;
  const uint32_t ex = a.mask_ex[w.z * kTile + lane];
  const uint32_t m14 = a.mask_14[w.z * kTile + lane];
  const bool valid_i = a.atom_valid[i] != 0;
  const double xi = a.x64[i], yi = a.y64[i], zi = a.z64[i], qi = a.q64[i], Ri = a.born_r64[i];
  const double rmi = a.rmin64[i], sepi = sqrt(a.eps64[i]), rm14i = a.rmin14_64[i], sep14i = sqrt(a.eps14_64[i]);
  const double iRi = 1.0 / Ri;
  const double coul_kj = kCoulomb * kKcalToKj;
  const double gb_pref = (1.0 - 1.0 / kEpsWater) * kCoulomb * kKcalToKj;
  const bool diag = w.x == w.y;
  double ax = 0.0, ay = 0.0, az = 0.0;
  __syncwarp();
  for (int k = diag ? 1 : 0; k < (diag ? 17 : kTile); ++k) {
    const int p = (lane + k) & (kTile - 1);
    double coeff = 0.0, dx = 0.0, dy = 0.0, dz = 0.0;
    if (valid_i && t.valid[p] && !(diag && k == 16 && lane >= 16)) {
      dx = t.x[p] - xi;
      dy = t.y[p] - yi;
      dz = t.z[p] - zi;
      const double r2 = dx * dx + dy * dy + dz * dz;
      const double qq = qi * t.q[p];
      if (r2 >= 1e-18) {
        // 1/r from one reciprocal square root; the GB factor
        // (1/f^2) ((2r - r e / 2) / (2f)) / r of the reference is
        // (1 - e/4) / f^3, and f^-1 another reciprocal square root
        const double inv_r = rsqrt(r2);
        const double inv_r2 = inv_r * inv_r;
        if (!((ex >> p) & 1u) && r2 <= a.nb_c2_64) {
          const bool is14 = (m14 >> p) & 1u;
          const double rmin = is14 ? rm14i + t.rmin14[p] : rmi + t.rmin[p];
          const double eps = is14 ? sep14i * t.seps14[p] : sepi * t.seps[p];
          const double ratio2 = rmin * rmin * inv_r2;
          const double r6 = ratio2 * ratio2 * ratio2;
          coeff += 12.0 * eps * inv_r2 * (r6 - r6 * r6) * kKcalToKj;
          if (qq != 0.0) coeff += -coul_kj * qq * (inv_r2 * inv_r - a.inv_rc3_64);
        }
        if (qq != 0.0 && r2 <= a.gb_c2_64) {
          const double rp = Ri * t.r[p];
          const double e = exp(-0.25 * r2 * (iRi * t.ir[p]));
          const double inv_f = rsqrt(r2 + rp * e);
          coeff += gb_pref * qq * (1.0 - 0.25 * e) * (inv_f * inv_f * inv_f);
        }
      }
    }
    ax += dx * coeff;
    ay += dy * coeff;
    az += dz * coeff;
    t.fx[p] -= dx * coeff;
    t.fy[p] -= dy * coeff;
    t.fz[p] -= dz * coeff;
    __syncwarp();
  }
  if (valid_i) {
    if (!(isfinite(ax) && isfinite(ay) && isfinite(az))) atomicOr(a.sys_nonfinite + a.atom_sys[i], 1);
    add_fixed(a.fx + i, ax, kForceScale);
    add_fixed(a.fy + i, ay, kForceScale);
    add_fixed(a.fz + i, az, kForceScale);
  }
  if (t.valid[lane]) {
    const double bx = t.fx[lane], by = t.fy[lane], bz = t.fz[lane];
    if (!(isfinite(bx) && isfinite(by) && isfinite(bz))) atomicOr(a.sys_nonfinite + a.atom_sys[jl], 1);
    add_fixed(a.fx + jl, bx, kForceScale);
    add_fixed(a.fy + jl, by, kForceScale);
    add_fixed(a.fz + jl, bz, kForceScale);
  }
}

}  // namespace

void launch_near_force64(const PairArgs& a, const int4* near, int n_near, cudaStream_t s) {
  if (n_near > 0) k_near64<<<(n_near + kNearWarps - 1) / kNearWarps, kNearWarps * 32, 0, s>>>(a, near, n_near);
}

// ----------------------------------------------------------------- FP64 path

namespace {

__device__ __forceinline__ double descreen64(double r, double rho_i, double s_rho_j) {
  // energy/src/gb.rs:347-369, term for term.
  if (r + s_rho_j <= rho_i) return 0.0;
  const double l = (r - s_rho_j < rho_i) ? rho_i : r - s_rho_j;
  const double u = r + s_rho_j;
  if (u <= 0.0 || l <= 0.0) return 0.0;
  const double inv_l = 1.0 / l, inv_u = 1.0 / u;
  const double term1 = 0.5 * (inv_l - inv_u);
  const double term2 = (r / 4.0) * (inv_u * inv_u - inv_l * inv_l);
  const double term3 = (1.0 / (2.0 * r)) * log(l / u);
  const double term4 = (s_rho_j * s_rho_j - r * r) / (4.0 * r) * (inv_u * inv_u - inv_l * inv_l);
  return term1 + term2 + term3 + term4;
}

// j range `c` of `nc` over a system's atoms [b, b + n).
__device__ __forceinline__ void chunk_range(int b, int n, int c, int nc, int* j0, int* j1) {
  *j0 = b + static_cast<int>(static_cast<long long>(n) * c / nc);
  *j1 = b + static_cast<int>(static_cast<long long>(n) * (c + 1) / nc);
}

__global__ void k_born64(EnergyArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = blockIdx.y;
  if (i >= a.n_atoms_padded) return;
  const int sys = a.atom_sys[i];
  if (sys < 0) return;
  int j0, j1;
  chunk_range(a.sys_begin[sys], a.sys_count[sys], c, a.n_chunks, &j0, &j1);
  const double xi = a.x[i], yi = a.y[i], zi = a.z[i], rho = a.rho_tilde[i];
  double acc = 0.0;
  for (int j = j0; j < j1; ++j) {
    if (j == i) continue;
    const double dx = a.x[j] - xi, dy = a.y[j] - yi, dz = a.z[j] - zi;
    const double r2 = dx * dx + dy * dy + dz * dz;
    if (r2 > a.born_c2 || r2 < 1e-18) continue;
    acc += descreen64(sqrt(r2), rho, a.srho[j]);
  }
  if (a.n_chunks == 1) a.integral[i] = acc;
  else a.part[static_cast<size_t>(c) * a.n_atoms_padded + i] = acc;
}

__global__ void k_born64_sum(EnergyArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n_atoms_padded || a.atom_sys[i] < 0) return;
  double acc = 0.0;
  for (int c = 0; c < a.n_chunks; ++c) acc += a.part[static_cast<size_t>(c) * a.n_atoms_padded + i];
  a.integral[i] = acc;
}

// Per i atom, over every j != i of its system: LJ + RF Coulomb within the
// nonbonded cutoff with exclusions / 1-4 parameters (nonbonded.rs:127-169)
// and the GB pair energy over all pairs (gb.rs:160-173).  Each unordered pair
// is seen from both ends, so the host halves the sums.
__global__ void k_energy64(EnergyArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = blockIdx.y;
  if (i >= a.n_atoms_padded) return;
  const int sys = a.atom_sys[i];
  const double pref = -0.5 * (1.0 - 1.0 / kEpsWater) * kCoulomb;
  if (sys < 0) {
    if (a.n_chunks == 1) {
      a.e_lj[i] = a.e_coul[i] = a.e_gb[i] = a.e_self[i] = 0.0;
      a.n_pairs[i] = 0;
    }
    return;
  }
  int j0, j1;
  chunk_range(a.sys_begin[sys], a.sys_count[sys], c, a.n_chunks, &j0, &j1);
  const double xi = a.x[i], yi = a.y[i], zi = a.z[i], qi = a.q[i], Ri = a.born_r[i];
  int ep = a.excl_row[i];
  const int ee = a.excl_row[i + 1];
  while (ep < ee && a.excl_col[ep] < j0) ++ep;
  double lj = 0.0, coul = 0.0, gb = 0.0;
  int pairs = 0;
  for (int j = j0; j < j1; ++j) {
    if (j == i) continue;
    const double dx = a.x[j] - xi, dy = a.y[j] - yi, dz = a.z[j] - zi;
    const double r2 = dx * dx + dy * dy + dz * dz;
    int kind = 0;
    while (ep < ee && a.excl_col[ep] < j) ++ep;
    if (ep < ee && a.excl_col[ep] == j) kind = a.excl_kind[ep];
    const double qq = qi * a.q[j];
    if (qq != 0.0) {
      // Once r2 / (4 rp) >= 40, rp exp(-r2 / (4 rp)) < r2 2^-54 (e^-40 <
      // 160 2^-54, and the gap only widens), below half an ulp of r2, so
      // r2 + rp exp(...) rounds to r2: the exponential is skipped there
      // with the same result bit for bit.
      const double rp = Ri * a.born_r[j];
      const double xg = r2 / (4.0 * rp);
      const double fgb = xg >= 40.0 ? sqrt(r2) : sqrt(r2 + rp * exp(-xg));
      gb += 2.0 * pref * qq / fgb;
    }
    if (r2 > a.nb_c2 || kind == 1) continue;
    const double r = sqrt(r2);
    double rmin, eps;
    if (kind == 2) {
      rmin = a.rmin14[i] + a.rmin14[j];
      eps = sqrt(a.eps14[i] * a.eps14[j]);
    } else {
      rmin = a.rmin[i] + a.rmin[j];
      eps = sqrt(a.eps[i] * a.eps[j]);
    }
    const double x = rmin / r;
    const double x2 = x * x;
    const double r6 = x2 * x2 * x2;
    lj += eps * (r6 * r6 - 2.0 * r6);
    if (qq != 0.0) coul += kCoulomb * qq * (1.0 / r + a.kappa * r * r - a.crf);
    ++pairs;
  }
  if (a.n_chunks == 1) {
    a.e_lj[i] = lj;
    a.e_coul[i] = coul;
    a.e_gb[i] = gb;
    a.e_self[i] = (qi != 0.0) ? pref * (qi * qi) / Ri : 0.0;
    a.n_pairs[i] = pairs;
    return;
  }
  const size_t np = a.n_atoms_padded, nc = a.n_chunks;
  a.part[(0 * nc + c) * np + i] = lj;
  a.part[(1 * nc + c) * np + i] = coul;
  a.part[(2 * nc + c) * np + i] = gb;
  a.part_pairs[c * np + i] = pairs;
}

__global__ void k_energy64_sum(EnergyArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n_atoms_padded) return;
  if (a.atom_sys[i] < 0) {
    a.e_lj[i] = a.e_coul[i] = a.e_gb[i] = a.e_self[i] = 0.0;
    a.n_pairs[i] = 0;
    return;
  }
  const size_t np = a.n_atoms_padded, nc = a.n_chunks;
  double lj = 0.0, coul = 0.0, gb = 0.0;
  int pairs = 0;
  for (size_t c = 0; c < nc; ++c) {
    lj += a.part[(0 * nc + c) * np + i];
    coul += a.part[(1 * nc + c) * np + i];
    gb += a.part[(2 * nc + c) * np + i];
    pairs += a.part_pairs[c * np + i];
  }
  const double pref = -0.5 * (1.0 - 1.0 / kEpsWater) * kCoulomb;
  const double qi = a.q[i];
  a.e_lj[i] = lj;
  a.e_coul[i] = coul;
  a.e_gb[i] = gb;
  a.e_self[i] = (qi != 0.0) ? pref * (qi * qi) / a.born_r[i] : 0.0;
  a.n_pairs[i] = pairs;
}

}  // namespace

void launch_born64(const EnergyArgs& a, cudaStream_t s) {
  const int bs = 128, nb = (a.n_atoms_padded + bs - 1) / bs;
  k_born64<<<dim3(nb, a.n_chunks), bs, 0, s>>>(a);
  if (a.n_chunks > 1) k_born64_sum<<<nb, bs, 0, s>>>(a);
}

void launch_energy64(const EnergyArgs& a, cudaStream_t s) {
  const int bs = 128, nb = (a.n_atoms_padded + bs - 1) / bs;
  k_energy64<<<dim3(nb, a.n_chunks), bs, 0, s>>>(a);
  if (a.n_chunks > 1) k_energy64_sum<<<nb, bs, 0, s>>>(a);
}

int energy_chunks(int n_atoms_padded, int max_system_atoms, int n_sm) {
  const int blocks = (n_atoms_padded + 127) / 128;
  int nc = (8 * n_sm + blocks - 1) / std::max(blocks, 1);
  nc = std::min(nc, std::max(1, max_system_atoms / 64));
  return std::max(1, std::min(nc, 32));
}

}  // namespace ogk
