// Pair kernels of the force path and the FP64 energy path.
//
// Force path (FP32 pair math):
//   born pass   -- descreening integral I_i = sum_j h(r_ij, rho~_i, s_j rho~_j)
//                  (energy/src/gb.rs:268-324 + pairwise_descreening :347-369)
//   force pass  -- LJ with 1-4 overrides + reaction-field Coulomb within the
//                  nonbonded cutoff (energy/src/forces_nonbonded.rs:196-232)
//                  fused with the frozen-radii GB pair force within the GB
//                  cutoff (energy/src/forces_gb.rs:82-111).
// Layout: one warp owns one 32-atom i-tile; a CTA of warps walks a list of
// 32-atom j-tiles that thread 0 streams into shared memory with 1-D TMA bulk
// copies (double buffered, mbarrier completion, bounded waits); each j atom
// is then read by all 32 lanes as a shared-memory broadcast.  The Born pass
// evaluates every ordered pair from its i side (h_ij and h_ji are different
// functions); the force pass evaluates each unordered far-field pair once and
// reduces the j-side force across the warp.  Every sum is formed in a fixed
// order (FP32 per j-tile, FP64 across tiles, 64-bit fixed point across work
// items), so results are bit-reproducible whatever the launch order.
//
// Positions reach the pair kernels as FP32 offsets from a per-tile FP64
// origin; the origin difference of a tile pair is formed in FP64 once per
// tile, which keeps |dx| accurate to ~1e-7 relative even for chains 1000 A
// long.
#include <cmath>

#include "common.cuh"
#include "pair_kernels.cuh"

namespace ogk {

namespace {

constexpr int kWarps = 4;         // i-tiles per CTA
constexpr int kStageTiles = 4;    // j-tiles per pipeline stage
constexpr float kLog2e = 1.4426950408889634f;

__device__ __forceinline__ float fast_rcp(float x) { return __fdividef(1.0f, x); }

// Born pass: h(r, rho_i, s_rho_j) summed over one staged j-tile.
//
// origami's pairwise_descreening (gb.rs:347-369) is
//   h = 1/2 (1/L - 1/U) + (r/4)(1/U^2 - 1/L^2) + ln(L/U)/(2r)
//       + (s^2 - r^2)/(4r) (1/U^2 - 1/L^2),      L = max(rho_i, r - s), U = r + s.
// Its terms cancel to O(s^3/r^4) for distant pairs, so FP32 evaluation of the
// closed form loses most digits there.  On the non-overlapping branch
// (L = r - s) the expression is, exactly, the series in x = s/r
//   h = -(x^3 / r) * sum_{k>=1} k(2k-1)/(2k+1) x^(2(k-1))
// (expand 1/(1-x^2), 1/(1-x^2)^2 and atanh x = -ln((1-x)/(1+x))/2 and collect
// powers).  For x < 1/4 eight terms leave a truncation error below 1e-8
// relative, under FP32 rounding.  A j atom takes that path when every lane's
// pair is distant (warp vote); otherwise all lanes use the closed form with
// term2 + term4 folded into (s^2 / 4r)(1/U^2 - 1/L^2) and
// ln(L/U) = log1p((L - U)/U).
constexpr float kSeriesMaxX = 0.25f;

__device__ __forceinline__ float descreen_series(float x, float inv_r) {
  const float x2 = x * x;
  float p = 120.0f / 17.0f;                 // k = 8
  p = fmaf(p, x2, 91.0f / 15.0f);           // k = 7
  p = fmaf(p, x2, 66.0f / 13.0f);           // k = 6
  p = fmaf(p, x2, 45.0f / 11.0f);           // k = 5
  p = fmaf(p, x2, 28.0f / 9.0f);            // k = 4
  p = fmaf(p, x2, 15.0f / 7.0f);            // k = 3
  p = fmaf(p, x2, 6.0f / 5.0f);             // k = 2
  p = fmaf(p, x2, 1.0f / 3.0f);             // k = 1
  return -(x2 * x * inv_r) * p;
}

// Closed form, valid on both branches.
__device__ __forceinline__ float descreen_closed(float r, float inv_r, float rho, float sr) {
  const bool overlap = (r - sr) < rho;
  const float L = overlap ? rho : r - sr;
  const float U = r + sr;
  const float inv_l = fast_rcp(L), inv_u = fast_rcp(U);
  const float lg = log1pf((overlap ? rho - U : -2.0f * sr) * inv_u);
  const float d2 = inv_u * inv_u - inv_l * inv_l;
  const float h = 0.5f * (inv_l - inv_u) + (sr * sr) * (0.25f * inv_r) * d2 + (0.5f * inv_r) * lg;
  return (!(r + sr <= rho) && (U > 0.0f) && (L > 0.0f)) ? h : 0.0f;
}

struct IAtom {
  float x, y, z;
  float cq;     // -coul_kj * q_i
  float gq;     // gb_pref_kj * q_i
  float rm;     // Rmin/2
  float se;     // 12 * 4.184 * sqrt(eps)
  float R;      // Born radius
  float nexp;   // -0.25 * log2(e) / R_i
};

}  // namespace


// ------------------------------------------------- far-field force, Newton-3
// Each unordered far-field tile pair (ti < tj, no masks) is evaluated once:
// the warp owning i-tile ti walks j-tile tj, every lane accumulates its i
// force in registers, and the force on each j atom (minus the sum over the
// 32 lanes) is formed by a butterfly reduction and kept by lane k for j = k.
// Per stage the W warps' j partials are summed in shared memory in a fixed
// order and added to the 64-bit fixed-point accumulators with one atomic per
// j atom and component, so results stay bit-reproducible.
namespace {

constexpr int kN3Warps = 8;

// Reduce-scatter over the warp of four per-lane values v0..v3 (the
// contributions to four consecutive j atoms): afterwards every lane of the
// 8-lane group g = lane >> 3 holds the warp total of v_g.  Six shuffles
// instead of the twenty of four separate butterflies; fixed order, so the
// result does not depend on scheduling.
__device__ __forceinline__ float reduce_scatter4(float v0, float v1, float v2, float v3, int lane) {
  const bool hi16 = (lane & 16) != 0;
  float k0 = hi16 ? v2 : v0, k1 = hi16 ? v3 : v1;   // kept: j = 2*hi16 + {0, 1}
  const float s0 = hi16 ? v0 : v2, s1 = hi16 ? v1 : v3;
  k0 += __shfl_xor_sync(0xffffffffu, s0, 16);
  k1 += __shfl_xor_sync(0xffffffffu, s1, 16);
  const bool hi8 = (lane & 8) != 0;
  float k = hi8 ? k1 : k0;                           // kept: j = 2*hi16 + hi8 = lane >> 3
  k += __shfl_xor_sync(0xffffffffu, hi8 ? k0 : k1, 8);
  k += __shfl_xor_sync(0xffffffffu, k, 4);
  k += __shfl_xor_sync(0xffffffffu, k, 2);
  k += __shfl_xor_sync(0xffffffffu, k, 1);
  return k;
}

template <bool kAllPairs>
__device__ __forceinline__ float pair_coeff(const float4 p, const float4 l, const float2 g, const IAtom& ia,
                                            const PairArgs& a, float dx, float dy, float dz) {
  const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
  const float inv_r = rsqrtf(r2);
  const float inv_r2 = inv_r * inv_r;
  const float rmin = ia.rm + l.x;
  const float ratio2 = rmin * rmin * inv_r2;
  const float r6 = ratio2 * ratio2 * ratio2;
  const float ljc = (ia.se * l.y) * inv_r2 * fmaf(-r6, r6, r6);       // ia.se carries 12 * 4.184
  const float coul = ia.cq * p.w * fmaf(inv_r2, inv_r, -a.inv_rc3);
  const float e = exp2f(r2 * ia.nexp * g.y);
  const float f2 = fmaf(ia.R * g.x, e, r2);
  const float inv_f = rsqrtf(f2);
  const float gbc = ia.gq * p.w * fmaf(-0.25f, e, 1.0f) * (inv_f * inv_f * inv_f);
  float coeff;
  if (kAllPairs) {
    coeff = ljc + coul + gbc;
  } else {
    coeff = ((r2 <= a.nb_c2) ? ljc + coul : 0.0f) + ((r2 <= a.gb_c2) ? gbc : 0.0f);
  }
  return (r2 >= 1e-18f) ? coeff : 0.0f;
}

template <bool kAllPairs>
__global__ void __launch_bounds__(kN3Warps * 32, 2) k_force_n3(PairArgs a) {
  constexpr uint32_t kTileBytes = kTile * sizeof(float4);
  constexpr int kStageAtoms = kStageTiles * kTile;
  __shared__ __align__(128) float4 s_buf[2][3][kStageAtoms];
  __shared__ float s_jf[kN3Warps][3][kStageAtoms];
  __shared__ __align__(8) uint64_t s_bar[2];

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const PairWork w = a.work[blockIdx.x];
  const int n_stages = (w.j_end - w.j_begin + kStageTiles - 1) / kStageTiles;

  if (threadIdx.x == 0) {
    mbar_init(&s_bar[0], 1);
    mbar_init(&s_bar[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  auto issue = [&](int s) {
    const int buf = s & 1;
    const int t0 = w.j_begin + s * kStageTiles;
    const int cnt = min(kStageTiles, w.j_end - t0);
    mbar_arrive_expect_tx(&s_bar[buf], static_cast<uint32_t>(cnt) * kTileBytes * 3);
    for (int t = 0; t < cnt; ++t) {
      const size_t base = static_cast<size_t>(a.jlist[t0 + t]) * kTile;
      bulk_g2s(&s_buf[buf][0][t * kTile], a.pq + base, kTileBytes, &s_bar[buf]);
      bulk_g2s(&s_buf[buf][1][t * kTile], a.lj + base, kTileBytes, &s_bar[buf]);
      bulk_g2s(&s_buf[buf][2][t * kTile], a.gb + base, kTileBytes, &s_bar[buf]);
    }
  };
  if (threadIdx.x == 0) {
    if (n_stages > 0) issue(0);
    if (n_stages > 1) issue(1);
  }

  const bool active = warp < w.n_i_tiles;
  const int it = w.i_tile0 + (active ? warp : 0);
  const int i = it * kTile + lane;
  const float4 pi = a.pq[i];
  const double4 oi = a.origin[it];
  IAtom ia;
  {
    const float4 li = a.lj[i];
    const float4 gi = a.gb[i];
    ia.cq = -a.coul_kj * pi.w;
    ia.gq = a.gb_pref_kj * pi.w;
    ia.rm = li.x;
    ia.se = a.lj_kj12 * li.y;
    ia.R = gi.x;
    ia.nexp = -0.25f * kLog2e * gi.y;
  }
  int mref = a.mask_begin[it];
  const int mend = a.mask_begin[it + 1];
  double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0;

  for (int s = 0; s < n_stages; ++s) {
    const int buf = s & 1;
    const bool ok = mbar_wait_bounded(&s_bar[buf], static_cast<uint32_t>((s >> 1) & 1));
    if (__syncthreads_or(!ok)) {
      if (threadIdx.x == 0) atomicOr(a.error_flag, kStatusTimeout);
      return;
    }
    const int t0 = w.j_begin + s * kStageTiles;
    const int cnt = min(kStageTiles, w.j_end - t0);
    for (int t = 0; t < cnt; ++t) {
      const int jt = a.jlist[t0 + t];
      while (mref < mend && a.mask_refs[mref].j_tile < jt) ++mref;
      const bool masked = mref < mend && a.mask_refs[mref].j_tile == jt;
      float* jfx = &s_jf[warp][0][t * kTile];
      float* jfy = &s_jf[warp][1][t * kTile];
      float* jfz = &s_jf[warp][2][t * kTile];
      if (active && jt > it && !masked) {
        const double4 oj = a.origin[jt];
        ia.x = pi.x - static_cast<float>(oj.x - oi.x);
        ia.y = pi.y - static_cast<float>(oj.y - oi.y);
        ia.z = pi.z - static_cast<float>(oj.z - oi.z);
        const float4* sp = &s_buf[buf][0][t * kTile];
        const float4* sl = &s_buf[buf][1][t * kTile];
        const float4* sg = &s_buf[buf][2][t * kTile];
        float fx = 0.0f, fy = 0.0f, fz = 0.0f;
#pragma unroll 2
        for (int k0 = 0; k0 < kTile; k0 += 4) {
          float ux[4], uy[4], uz[4];
#pragma unroll
          for (int g = 0; g < 4; ++g) {
            const int k = k0 + g;
            const float4 p = sp[k];
            const float4 l = sl[k];
            const float2 gg = *reinterpret_cast<const float2*>(&sg[k]);
            const float dx = p.x - ia.x, dy = p.y - ia.y, dz = p.z - ia.z;
            const float c = pair_coeff<kAllPairs>(p, l, gg, ia, a, dx, dy, dz);
            ux[g] = dx * c;
            uy[g] = dy * c;
            uz[g] = dz * c;
            fx += ux[g];
            fy += uy[g];
            fz += uz[g];
          }
          const float tx = reduce_scatter4(ux[0], ux[1], ux[2], ux[3], lane);
          const float ty = reduce_scatter4(uy[0], uy[1], uy[2], uy[3], lane);
          const float tz = reduce_scatter4(uz[0], uz[1], uz[2], uz[3], lane);
          if ((lane & 7) == 0) {
            jfx[k0 + (lane >> 3)] = -tx;
            jfy[k0 + (lane >> 3)] = -ty;
            jfz[k0 + (lane >> 3)] = -tz;
          }
        }
        acc0 += static_cast<double>(fx);
        acc1 += static_cast<double>(fy);
        acc2 += static_cast<double>(fz);
      } else {
        jfx[lane] = 0.0f;
        jfy[lane] = 0.0f;
        jfz[lane] = 0.0f;
      }
    }
    __syncthreads();  // every warp is done with `buf` and has written its j partials
    if (threadIdx.x == 0 && s + 2 < n_stages) issue(s + 2);
    for (int q = threadIdx.x; q < cnt * kTile; q += blockDim.x) {
      const int j = a.jlist[t0 + q / kTile] * kTile + (q % kTile);
      if (!a.atom_valid[j]) continue;
      float sx = 0.0f, sy = 0.0f, sz = 0.0f;
#pragma unroll
      for (int ww = 0; ww < kN3Warps; ++ww) {
        sx += s_jf[ww][0][q];
        sy += s_jf[ww][1][q];
        sz += s_jf[ww][2][q];
      }
      if (sx != 0.0f || sy != 0.0f || sz != 0.0f) {
        if (!(isfinite(sx) && isfinite(sy) && isfinite(sz))) atomicOr(a.sys_nonfinite + a.atom_sys[j], 1);
        add_fixed(a.fx + j, sx, kForceScale);
        add_fixed(a.fy + j, sy, kForceScale);
        add_fixed(a.fz + j, sz, kForceScale);
      }
    }
  }
  if (active && a.atom_valid[i]) {
    if (!(isfinite(acc0) && isfinite(acc1) && isfinite(acc2))) atomicOr(a.sys_nonfinite + a.atom_sys[i], 1);
    add_fixed(a.fx + i, acc0, kForceScale);
    add_fixed(a.fy + i, acc1, kForceScale);
    add_fixed(a.fz + i, acc2, kForceScale);
  }
}


// ------------------------------------------------------ Born pass, Newton-3
// Each unordered tile pair (ti <= tj) is visited once: h_ij feeds atom i
// (lane registers) and h_ji feeds atom j (reduce-scatter across the warp,
// then a fixed-order sum over warps in shared memory).  The distance is
// shared by both directions.  The diagonal tile is evaluated from the i
// side only, over all ordered pairs.
__device__ __forceinline__ float born_pair(float r, float inv_r, float rho, float sr, bool series) {
  return series ? descreen_series(sr * inv_r, inv_r) : descreen_closed(r, inv_r, rho, sr);
}

__global__ void __launch_bounds__(kN3Warps * 32) k_born_n3(PairArgs a) {
  constexpr uint32_t kTileBytes = kTile * sizeof(float4);
  constexpr int kStageAtoms = kStageTiles * kTile;
  __shared__ __align__(128) float4 s_buf[2][2][kStageAtoms];
  __shared__ float s_jh[kN3Warps][kStageAtoms];
  __shared__ __align__(8) uint64_t s_bar[2];

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const PairWork w = a.work[blockIdx.x];
  const int n_stages = (w.j_end - w.j_begin + kStageTiles - 1) / kStageTiles;
  if (threadIdx.x == 0) {
    mbar_init(&s_bar[0], 1);
    mbar_init(&s_bar[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  auto issue = [&](int s) {
    const int buf = s & 1;
    const int t0 = w.j_begin + s * kStageTiles;
    const int cnt = min(kStageTiles, w.j_end - t0);
    mbar_arrive_expect_tx(&s_bar[buf], static_cast<uint32_t>(cnt) * kTileBytes * 2);
    for (int t = 0; t < cnt; ++t) {
      const size_t base = static_cast<size_t>(a.jlist[t0 + t]) * kTile;
      bulk_g2s(&s_buf[buf][0][t * kTile], a.pq + base, kTileBytes, &s_bar[buf]);
      bulk_g2s(&s_buf[buf][1][t * kTile], a.gb + base, kTileBytes, &s_bar[buf]);
    }
  };
  if (threadIdx.x == 0) {
    if (n_stages > 0) issue(0);
    if (n_stages > 1) issue(1);
  }

  const bool active = warp < w.n_i_tiles;
  const int it = w.i_tile0 + (active ? warp : 0);
  const int i = it * kTile + lane;
  const float4 pi = a.pq[i];
  const double4 oi = a.origin[it];
  const float rho_i = a.gb[i].z, s_i = a.gb[i].w;
  const float c2 = a.born_c2;
  double acc = 0.0;
  for (int s = 0; s < n_stages; ++s) {
    const int buf = s & 1;
    const bool ok = mbar_wait_bounded(&s_bar[buf], static_cast<uint32_t>((s >> 1) & 1));
    if (__syncthreads_or(!ok)) {
      if (threadIdx.x == 0) atomicOr(a.error_flag, kStatusTimeout);
      return;
    }
    const int t0 = w.j_begin + s * kStageTiles;
    const int cnt = min(kStageTiles, w.j_end - t0);
    for (int t = 0; t < cnt; ++t) {
      const int jt = a.jlist[t0 + t];
      float* jh = &s_jh[warp][t * kTile];
      if (!active || jt < it) {
        jh[lane] = 0.0f;
        continue;
      }
      const double4 oj = a.origin[jt];
      const float xi = pi.x - static_cast<float>(oj.x - oi.x);
      const float yi = pi.y - static_cast<float>(oj.y - oi.y);
      const float zi = pi.z - static_cast<float>(oj.z - oi.z);
      const float4* sp = &s_buf[buf][0][t * kTile];
      const float4* sg = &s_buf[buf][1][t * kTile];
      float hi_acc = 0.0f;
      if (jt == it) {
#pragma unroll 4
        for (int k = 0; k < kTile; ++k) {
          const float4 p = sp[k];
          const float sr = sg[k].w;
          const float dx = p.x - xi, dy = p.y - yi, dz = p.z - zi;
          const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
          const float inv_r = rsqrtf(r2);
          const float r = r2 * inv_r;
          const bool far = (sr * inv_r < kSeriesMaxX) && (r - sr >= rho_i);
          const float h = born_pair(r, inv_r, rho_i, sr, __all_sync(0xffffffffu, far));
          hi_acc += ((r2 <= c2) && (r2 >= 1e-18f)) ? h : 0.0f;
        }
        jh[lane] = 0.0f;
      } else {
#pragma unroll 2
        for (int k0 = 0; k0 < kTile; k0 += 4) {
          float u[4];
#pragma unroll
          for (int g = 0; g < 4; ++g) {
            const int k = k0 + g;
            const float4 p = sp[k];
            const float4 gj = sg[k];  // rho~_j in z, s_j rho~_j in w
            const float dx = p.x - xi, dy = p.y - yi, dz = p.z - zi;
            const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            const float inv_r = rsqrtf(r2);
            const float r = r2 * inv_r;
            const bool far = (gj.w * inv_r < kSeriesMaxX) && (s_i * inv_r < kSeriesMaxX) && (r - gj.w >= rho_i) &&
                             (r - s_i >= gj.z);
            const bool series = __all_sync(0xffffffffu, far);
            const bool on = (r2 <= c2) && (r2 >= 1e-18f);
            const float hij = born_pair(r, inv_r, rho_i, gj.w, series);
            const float hji = born_pair(r, inv_r, gj.z, s_i, series);
            hi_acc += on ? hij : 0.0f;
            u[g] = on ? hji : 0.0f;
          }
          const float tot = reduce_scatter4(u[0], u[1], u[2], u[3], lane);
          if ((lane & 7) == 0) jh[k0 + (lane >> 3)] = tot;
        }
      }
      acc += static_cast<double>(hi_acc);
    }
    __syncthreads();  // every warp is done with `buf` and has written its j partials
    if (threadIdx.x == 0 && s + 2 < n_stages) issue(s + 2);
    for (int q = threadIdx.x; q < cnt * kTile; q += blockDim.x) {
      const int j = a.jlist[t0 + q / kTile] * kTile + (q % kTile);
      if (!a.atom_valid[j]) continue;
      float sum = 0.0f;
#pragma unroll
      for (int ww = 0; ww < kN3Warps; ++ww) sum += s_jh[ww][q];
      if (sum != 0.0f) {
        if (!isfinite(sum)) atomicOr(a.sys_nonfinite + a.atom_sys[j], 1);
        add_fixed(a.born_sum + j, static_cast<double>(sum), kBornScale);
      }
    }
  }
  if (active && a.atom_valid[i]) {
    if (!isfinite(acc)) atomicOr(a.sys_nonfinite + a.atom_sys[i], 1);
    add_fixed(a.born_sum + i, acc, kBornScale);
  }
}

}  // namespace

int force_warps_per_cta() { return kN3Warps; }

void launch_born_pass(const PairArgs& a, cudaStream_t s) {
  if (a.n_work > 0) k_born_n3<<<a.n_work, kN3Warps * 32, 0, s>>>(a);
}

void launch_force_pass(const PairArgs& a, cudaStream_t s) {
  if (a.n_work <= 0) return;
  if (a.nb_c2 == INFINITY && a.gb_c2 == INFINITY)
    k_force_n3<true><<<a.n_work, kN3Warps * 32, 0, s>>>(a);
  else
    k_force_n3<false><<<a.n_work, kN3Warps * 32, 0, s>>>(a);
}

int pair_warps_per_cta() { return kWarps; }

// ------------------------------------------------------- FP64 near field
// One warp per near-field (i-tile, j-tile) pair -- the tiles that carry
// exclusion / 1-4 masks, i.e. the bonded neighbourhood where the large LJ and
// Coulomb pair forces cancel against the bonded terms.  FP64 throughout, term
// for term as forces_nonbonded.rs:196-232 + forces_gb.rs:82-111; the j atoms
// are warp-uniform broadcast loads.
namespace {

__global__ void __launch_bounds__(128) k_near64(PairArgs a, const int4* __restrict__ near, int n_near) {
  const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (wid >= n_near) return;
  const int4 w = near[wid];  // i_tile, j_tile, mask offset
  const int i = w.x * kTile + lane;
  const uint32_t ex = a.mask_ex[w.z * kTile + lane];
  const uint32_t m14 = a.mask_14[w.z * kTile + lane];
  const double xi = a.x64[i], yi = a.y64[i], zi = a.z64[i], qi = a.q64[i], Ri = a.born_r64[i];
  const double rmi = a.rmin64[i], epi = a.eps64[i], rm14i = a.rmin14_64[i], ep14i = a.eps14_64[i];
  const double coul_kj = kCoulomb * kKcalToKj;
  const double gb_pref = (1.0 - 1.0 / kEpsWater) * kCoulomb * kKcalToKj;
  double ax = 0.0, ay = 0.0, az = 0.0;
  const int j0 = w.y * kTile;
  for (int k = 0; k < kTile; ++k) {
    const int j = j0 + k;
    if (!a.atom_valid[j]) continue;
    const double dx = a.x64[j] - xi, dy = a.y64[j] - yi, dz = a.z64[j] - zi;
    const double r2 = dx * dx + dy * dy + dz * dz;
    if (r2 < 1e-18) continue;
    const double qq = qi * a.q64[j];
    double coeff = 0.0;
    if (!((ex >> k) & 1u) && r2 <= a.nb_c2_64) {
      const bool is14 = (m14 >> k) & 1u;
      const double rmin = is14 ? rm14i + a.rmin14_64[j] : rmi + a.rmin64[j];
      const double eps = sqrt(is14 ? ep14i * a.eps14_64[j] : epi * a.eps64[j]);
      const double inv_r2 = 1.0 / r2;
      const double ratio2 = rmin * rmin * inv_r2;
      const double r6 = ratio2 * ratio2 * ratio2;
      coeff += 12.0 * eps * inv_r2 * (r6 - r6 * r6) * kKcalToKj;
      if (qq != 0.0) coeff += -coul_kj * qq * (inv_r2 / sqrt(r2) - a.inv_rc3_64);
    }
    if (qq != 0.0 && r2 <= a.gb_c2_64) {
      const double r = sqrt(r2);
      const double rp = Ri * a.born_r64[j];
      const double e = exp(-r2 / (4.0 * rp));
      const double f2 = r2 + rp * e;
      const double f = sqrt(f2);
      coeff += gb_pref * qq / f2 * ((2.0 * r - 0.5 * r * e) / (2.0 * f)) / r;
    }
    ax += dx * coeff;
    ay += dy * coeff;
    az += dz * coeff;
  }
  if (a.atom_valid[i]) {
    if (!(isfinite(ax) && isfinite(ay) && isfinite(az))) atomicOr(a.sys_nonfinite + a.atom_sys[i], 1);
    add_fixed(a.fx + i, ax, kForceScale);
    add_fixed(a.fy + i, ay, kForceScale);
    add_fixed(a.fz + i, az, kForceScale);
  }
}

}  // namespace

void launch_near_force64(const PairArgs& a, const int4* near, int n_near, cudaStream_t s) {
  if (n_near > 0) k_near64<<<(n_near * 32 + 127) / 128, 128, 0, s>>>(a, near, n_near);
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

__global__ void k_born64(EnergyArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n_atoms_padded) return;
  const int sys = a.atom_sys[i];
  if (sys < 0) return;
  const int b = a.sys_begin[sys], n = a.sys_count[sys];
  const double xi = a.x[i], yi = a.y[i], zi = a.z[i], rho = a.rho_tilde[i];
  double acc = 0.0;
  for (int j = b; j < b + n; ++j) {
    if (j == i) continue;
    const double dx = a.x[j] - xi, dy = a.y[j] - yi, dz = a.z[j] - zi;
    const double r2 = dx * dx + dy * dy + dz * dz;
    if (r2 > a.born_c2 || r2 < 1e-18) continue;
    acc += descreen64(sqrt(r2), rho, a.srho[j]);
  }
  a.integral[i] = acc;
}

// Per i atom, over every j != i of its system: LJ + RF Coulomb within the
// nonbonded cutoff with exclusions / 1-4 parameters (nonbonded.rs:127-169)
// and the GB pair energy over all pairs (gb.rs:160-173).  Each unordered pair
// is seen from both ends, so the host halves the sums.
__global__ void k_energy64(EnergyArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n_atoms_padded) return;
  const int sys = a.atom_sys[i];
  if (sys < 0) {
    a.e_lj[i] = a.e_coul[i] = a.e_gb[i] = a.e_self[i] = 0.0;
    a.n_pairs[i] = 0;
    return;
  }
  const int b = a.sys_begin[sys], n = a.sys_count[sys];
  const double xi = a.x[i], yi = a.y[i], zi = a.z[i], qi = a.q[i], Ri = a.born_r[i];
  const double pref = -0.5 * (1.0 - 1.0 / kEpsWater) * kCoulomb;
  int ep = a.excl_row[i];
  const int ee = a.excl_row[i + 1];
  double lj = 0.0, coul = 0.0, gb = 0.0;
  int pairs = 0;
  for (int j = b; j < b + n; ++j) {
    if (j == i) continue;
    const double dx = a.x[j] - xi, dy = a.y[j] - yi, dz = a.z[j] - zi;
    const double r2 = dx * dx + dy * dy + dz * dz;
    int kind = 0;
    while (ep < ee && a.excl_col[ep] < j) ++ep;
    if (ep < ee && a.excl_col[ep] == j) kind = a.excl_kind[ep];
    const double qq = qi * a.q[j];
    if (qq != 0.0) {
      const double rp = Ri * a.born_r[j];
      const double fgb = sqrt(r2 + rp * exp(-r2 / (4.0 * rp)));
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
  a.e_lj[i] = lj;
  a.e_coul[i] = coul;
  a.e_gb[i] = gb;
  a.e_self[i] = (qi != 0.0) ? pref * (qi * qi) / Ri : 0.0;
  a.n_pairs[i] = pairs;
}

}  // namespace

void launch_born64(const EnergyArgs& a, cudaStream_t s) {
  const int bs = 128;
  k_born64<<<(a.n_atoms_padded + bs - 1) / bs, bs, 0, s>>>(a);
}

void launch_energy64(const EnergyArgs& a, cudaStream_t s) {
  const int bs = 128;
  k_energy64<<<(a.n_atoms_padded + bs - 1) / bs, bs, 0, s>>>(a);
}

}  // namespace ogk
