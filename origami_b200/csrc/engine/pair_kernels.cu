// FP32 tiled pair kernels of the force path.
//
//   born pass   -- descreening integral I_i = sum_j h(r_ij, rho~_i, s_j rho~_j)
//                  (energy/src/gb.rs:268-324 + pairwise_descreening :347-369)
//   force pass  -- LJ + reaction-field Coulomb within the nonbonded cutoff
//                  (energy/src/forces_nonbonded.rs:196-232) fused with the
//                  frozen-radii GB pair force within the GB cutoff
//                  (energy/src/forces_gb.rs:82-111), far-field tiles only;
//                  near-field tiles (exclusions, 1-4 pairs) go to the FP64
//                  kernel in pair_fp64.cu.
//
// Layout.  One warp owns one 32-atom i-tile and a CTA of W warps owns W
// consecutive tiles (W = 8 or 4, a launch variant).  The CTA walks a list of
// j-tiles (the tiles from
// its first tile on -- each unordered tile pair once); thread 0 streams them
// into shared memory with 1-D TMA bulk copies (two stages in flight, mbarrier
// completion, bounded waits).  The per-atom FP32 arrays are tile-SoA (four
// 32-float columns per tile), so one 16-byte shared load is one column of
// four consecutive j atoms, which feeds Blackwell's packed FP32x2 arithmetic
// directly: the force pass evaluates two j atoms per instruction, the Born
// pass the two directions h_ij / h_ji of one pair.  The j-side sums (Newton's
// third law) are formed by a warp reduce-scatter, summed over the CTA's warps
// in shared memory in a fixed order and added to 64-bit fixed-point
// accumulators; the i side accumulates FP32 per tile and FP64 across tiles.
// Every sum therefore has a fixed order and results are bit-reproducible.
//
// Launch variants (PairConfig): W, the CTAs per SM the register budget is
// sized for, and either one CTA per work item (the hardware assigns CTAs to
// SMs as they free up) or a persistent grid of resident CTAs that take items
// from an atomic queue.  The engine's autotuner times them on the actual
// systems; every variant computes the same sums in the same order.
//
// Positions are FP32 offsets from a per-tile FP64 origin; the origin
// difference of a tile pair is formed in FP64 once per tile, so |dx| keeps
// ~1e-7 relative accuracy in chains 1000 A long.
#include <algorithm>
#include <cmath>

#include "common.cuh"
#include "pair_kernels.cuh"

namespace ogk {

namespace {

// Groups of four j atoms in flight per lane (measured best on B200 for
// 64 x 4.7k-atom systems).
#ifndef OG_BORN_UNROLL
#define OG_BORN_UNROLL 1
#endif
#ifndef OG_FORCE_UNROLL
#define OG_FORCE_UNROLL 2
#endif
#define OG_PRAGMA(x) _Pragma(#x)
#define OG_UNROLL(n) OG_PRAGMA(unroll n)

constexpr int kStageTiles = 4;    // j-tiles per pipeline stage
constexpr int kStageFloats = kStageTiles * 128;
constexpr uint32_t kTileBytes = 128 * sizeof(float);
constexpr float kLog2e = 1.4426950408889634f;

__device__ __forceinline__ float2 bc(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float fast_rcp(float x) { return __fdividef(1.0f, x); }

// Reduce-scatter over the warp of four per-lane values v0..v3 (contributions
// to four consecutive j atoms): afterwards every lane of the 8-lane group
// g = lane >> 3 holds the warp total of v_g.  Six shuffles instead of the
// twenty of four separate butterflies; the order is fixed.
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

// ------------------------------------------------------------- staging
// Stage s of a work item is the CTA's stage g0 + s overall: buffer and
// mbarrier (g0 + s) & 1, wait parity ((g0 + s) >> 1) & 1, so a persistent
// CTA keeps alternating its two barriers across items.
template <int kST = kStageTiles>
struct StagerT {
  const int32_t* jlist;
  int j_begin, j_end, n_stages;
  uint64_t* bar;
  uint32_t g0;
  template <int kArrays>
  __device__ __forceinline__ void issue(int s, float (*buf)[kArrays][kST * 128], const float* const* src) const {
    const int b = (g0 + s) & 1;
    const int t0 = j_begin + s * kST;
    const int cnt = min(kST, j_end - t0);
    mbar_arrive_expect_tx(&bar[b], static_cast<uint32_t>(cnt) * kTileBytes * kArrays);
    for (int t = 0; t < cnt; ++t) {
      const size_t base = static_cast<size_t>(jlist[t0 + t]) * 128;
#pragma unroll
      for (int c = 0; c < kArrays; ++c) bulk_g2s(&buf[b][c][t * 128], src[c] + base, kTileBytes, &bar[b]);
    }
  }
};

using Stager = StagerT<>;

// Adds the stage's j partials (s_part[w][c][q], summed over warps in a fixed
// order) to the fixed-point accumulators.
template <int W, int kComps, int kST = kStageTiles>
__device__ __forceinline__ void flush_j(const PairArgs& a, const int32_t* jlist, int t0, int cnt,
                                        float (*s_part)[kComps][kST * kTile], unsigned long long* const* dst,
                                        double scale) {
  for (int q = threadIdx.x; q < cnt * kTile; q += blockDim.x) {
    const int j = jlist[t0 + q / kTile] * kTile + (q % kTile);
    if (!a.atom_valid[j]) continue;
    float v[kComps];
    bool any = false, finite = true;
#pragma unroll
    for (int c = 0; c < kComps; ++c) {
      float sum = 0.0f;
#pragma unroll
      for (int w = 0; w < W; ++w) sum += s_part[w][c][q];
      v[c] = sum;
      any = any || sum != 0.0f;
      finite = finite && isfinite(sum);
    }
    if (!any) continue;
    if (!finite) atomicOr(a.sys_nonfinite + a.atom_sys[j], 1);
#pragma unroll
    for (int c = 0; c < kComps; ++c) add_fixed(dst[c] + j, static_cast<double>(v[c]), scale);
  }
}

// ---------------------------------------------------------------- Born
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
// pair is distant in both directions (warp vote); otherwise all lanes use the
// closed form with term2 + term4 folded into (s^2 / 4r)(1/U^2 - 1/L^2) and
// ln(L/U) = log1p((L - U)/U).
constexpr float kSeriesMaxX = 0.25f;

// Series for the two directions at once: x = (s_j, s_i) / r.
__device__ __forceinline__ float2 descreen_series2(float2 x, float inv_r) {
  const float2 xx = mul2(x, x);
  float2 p = bc(120.0f / 17.0f);
  p = fma2(p, xx, bc(91.0f / 15.0f));
  p = fma2(p, xx, bc(66.0f / 13.0f));
  p = fma2(p, xx, bc(45.0f / 11.0f));
  p = fma2(p, xx, bc(28.0f / 9.0f));
  p = fma2(p, xx, bc(15.0f / 7.0f));
  p = fma2(p, xx, bc(6.0f / 5.0f));
  p = fma2(p, xx, bc(1.0f / 3.0f));
  return mul2(mul2(mul2(xx, x), bc(-inv_r)), p);
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

// (h_ij, h_ji) for one pair; on = inside the Born cutoff and not coincident.
__device__ __forceinline__ float2 born_pair(float dx, float dy, float dz, float rho_i, float s_i, float rho_j,
                                           float s_j, float c2) {
  const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
  const float inv_r = rsqrtf(r2);
  const float r = r2 * inv_r;
  const float2 x = mul2(make_float2(s_j, s_i), bc(inv_r));
  const bool far = (x.x < kSeriesMaxX) && (x.y < kSeriesMaxX) && (r - s_j >= rho_i) && (r - s_i >= rho_j);
  float2 h;
  if (__all_sync(0xffffffffu, far)) {
    h = descreen_series2(x, inv_r);
  } else {
    h = make_float2(descreen_closed(r, inv_r, rho_i, s_j), descreen_closed(r, inv_r, rho_j, s_i));
  }
  const bool on = (r2 <= c2) && (r2 >= 1e-18f);
  return on ? h : make_float2(0.0f, 0.0f);
}

// The next work item of a CTA: its own (one CTA per item) or the queue's.
template <bool kPersistent>
__device__ __forceinline__ int next_item(const PairArgs& a, int* s_item, int prev) {
  if (!kPersistent) return prev < 0 ? static_cast<int>(blockIdx.x) : a.n_work;
  __syncthreads();  // every thread has read the previous item
  if (threadIdx.x == 0) *s_item = atomicAdd(a.queue, 1);
  __syncthreads();
  return *s_item;
}

template <int W, int kMinBlocks, bool kPersistent>
__global__ void __launch_bounds__(W * 32, kMinBlocks) k_born(PairArgs a) {
  __shared__ __align__(128) float s_buf[2][2][kStageFloats];          // columns of pq, gb
  __shared__ float s_part[W][1][kStageTiles * kTile];
  __shared__ __align__(8) uint64_t s_bar[2];
  __shared__ int s_item;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    mbar_init(&s_bar[0], 1);
    mbar_init(&s_bar[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  uint32_t g = 0;  // stages this CTA has consumed
  for (int item = next_item<kPersistent>(a, &s_item, -1); item < a.n_work;
       item = next_item<kPersistent>(a, &s_item, item)) {
  PairWork w = a.work[item];
  if (a.seg_end) w.j_end = min(w.j_end, a.seg_end[w.i_tile0]);
  if (w.j_begin >= w.j_end) continue;  // chunk culled by the cutoff (block-uniform)
  const Stager st{a.jlist, w.j_begin, w.j_end, (w.j_end - w.j_begin + kStageTiles - 1) / kStageTiles, s_bar, g};
  const float* src[2] = {a.pq, a.gb};
  if (threadIdx.x == 0) {
    if (st.n_stages > 0) st.issue<2>(0, s_buf, src);
    if (st.n_stages > 1) st.issue<2>(1, s_buf, src);
  }

  const bool active = warp < w.n_i_tiles;
  const int it = w.i_tile0 + (active ? warp : 0);
  const int i = it * kTile + lane;
  const float px = a.pq[soa_index(i, 0)], py = a.pq[soa_index(i, 1)], pz = a.pq[soa_index(i, 2)];
  const float rho_i = a.gb[soa_index(i, 2)], s_i = a.gb[soa_index(i, 3)];
  const double4 oi = a.origin[it];
  const float c2 = a.born_c2;
  double acc = 0.0;
  for (int s = 0; s < st.n_stages; ++s) {
    const uint32_t gs = g + s;
    const int b = gs & 1;
    const bool ok = mbar_wait_bounded(&s_bar[b], (gs >> 1) & 1u);
    if (__syncthreads_or(!ok)) {
      if (threadIdx.x == 0) atomicOr(a.error_flag, kStatusTimeout);
      return;
    }
    const int t0 = w.j_begin + s * kStageTiles;
    const int cnt = min(kStageTiles, w.j_end - t0);
    for (int t = 0; t < cnt; ++t) {
      const int jt = a.jlist[t0 + t];
      float* part = &s_part[warp][0][t * kTile];
      if (!active || jt < it) {
        part[lane] = 0.0f;
        continue;
      }
      const double4 oj = a.origin[jt];
      const float xi = px - static_cast<float>(oj.x - oi.x);
      const float yi = py - static_cast<float>(oj.y - oi.y);
      const float zi = pz - static_cast<float>(oj.z - oi.z);
      const float* sp = &s_buf[b][0][t * 128];
      const float* sg = &s_buf[b][1][t * 128];
      float hi = 0.0f;
      if (jt == it) {
        // Diagonal tile: every ordered pair from the i side.
#pragma unroll 4
        for (int k = 0; k < kTile; ++k) {
          const float2 h = born_pair(sp[k] - xi, sp[32 + k] - yi, sp[64 + k] - zi, rho_i, s_i, sg[64 + k],
                                     sg[96 + k], c2);
          hi += h.x;
        }
        part[lane] = 0.0f;
      } else {
OG_UNROLL(OG_BORN_UNROLL)
        for (int k0 = 0; k0 < kTile; k0 += 4) {
          const float4 X = *reinterpret_cast<const float4*>(&sp[k0]);
          const float4 Y = *reinterpret_cast<const float4*>(&sp[32 + k0]);
          const float4 Z = *reinterpret_cast<const float4*>(&sp[64 + k0]);
          const float4 RH = *reinterpret_cast<const float4*>(&sg[64 + k0]);
          const float4 SR = *reinterpret_cast<const float4*>(&sg[96 + k0]);
          const float2 h0 = born_pair(X.x - xi, Y.x - yi, Z.x - zi, rho_i, s_i, RH.x, SR.x, c2);
          const float2 h1 = born_pair(X.y - xi, Y.y - yi, Z.y - zi, rho_i, s_i, RH.y, SR.y, c2);
          const float2 h2 = born_pair(X.z - xi, Y.z - yi, Z.z - zi, rho_i, s_i, RH.z, SR.z, c2);
          const float2 h3 = born_pair(X.w - xi, Y.w - yi, Z.w - zi, rho_i, s_i, RH.w, SR.w, c2);
          hi += (h0.x + h1.x) + (h2.x + h3.x);
          const float tot = reduce_scatter4(h0.y, h1.y, h2.y, h3.y, lane);
          if ((lane & 7) == 0) part[k0 + (lane >> 3)] = tot;
        }
      }
      acc += static_cast<double>(hi);
    }
    __syncthreads();  // every warp is done with buffer b and has written its j partials
    if (threadIdx.x == 0 && s + 2 < st.n_stages) st.issue<2>(s + 2, s_buf, src);
    unsigned long long* dst[1] = {a.born_sum};
    flush_j<W, 1>(a, a.jlist, t0, cnt, s_part, dst, kBornScale);
  }
  g += st.n_stages;
  if (active && a.atom_valid[i]) {
    if (!isfinite(acc)) atomicOr(a.sys_nonfinite + a.atom_sys[i], 1);
    add_fixed(a.born_sum + i, acc, kBornScale);
  }
  }
}

// --------------------------------------------------------------- force
// i-atom data broadcast into both halves of a float2.
struct IAtom2 {
  float2 nx, ny, nz;   // minus the i position relative to the j-tile's origin
  float2 rm;           // Rmin/2
  float2 se;           // 12 * 4.184 * sqrt(eps)
  float2 cq;           // -332.0637 * 4.184 * q_i
  float2 gq;           // (1 - 1/78.5) * 332.0637 * 4.184 * q_i
  float2 R;            // Born radius
  float2 nexp;         // -log2(e) / (4 R_i)
  float2 nrc3;         // -1 / Rc^3
};

// Separation d = x_j - x_i of two j atoms from the i atom, and r^2.
struct Sep2 {
  float2 dx, dy, dz, r2;
};
__device__ __forceinline__ Sep2 sep2(float2 xj, float2 yj, float2 zj, const IAtom2& ia) {
  Sep2 s;
  s.dx = add2(xj, ia.nx);
  s.dy = add2(yj, ia.ny);
  s.dz = add2(zj, ia.nz);
  s.r2 = fma2(s.dx, s.dx, fma2(s.dy, s.dy, mul2(s.dz, s.dz)));
  return s;
}

// Exponent of the GB kernel's exponential in base 2: -r^2 / (4 R_i R_j) log2(e).
__device__ __forceinline__ float2 gb_arg2(const Sep2& s, float2 iRj, const IAtom2& ia) {
  return mul2(mul2(s.r2, ia.nexp), iRj);
}

// Pair coefficients c (F_i = c * d) for two j atoms.  kFarGb: both pairs
// have arg < -30, so e = 2^arg < 2^-30: R_i R_j e < r^2 / 83 * 2^-30 is below
// half an ulp of r^2, so f^2 = fma(R_i R_j, e, r^2) rounds to r^2 and
// 1 - e/4 to 1; the far form then evaluates exactly what the full form does
// (same rsqrt input, same products), without the exponential and the
// second reciprocal square root.
template <bool kAllPairs, bool kFarGb>
__device__ __forceinline__ float2 coeff2(const Sep2& s, float2 arg, float2 qj, float2 rmj, float2 sej, float2 Rj,
                                         const IAtom2& ia, const PairArgs& a) {
  const float2 r2 = s.r2;
  const float2 inv_r = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
  const float2 inv_r2 = mul2(inv_r, inv_r);
  const float2 rmin = add2(ia.rm, rmj);
  const float2 ratio2 = mul2(mul2(rmin, rmin), inv_r2);
  const float2 r6 = mul2(mul2(ratio2, ratio2), ratio2);
  const float2 one_m_r6 = fma2(r6, bc(-1.0f), bc(1.0f));
  const float2 ljc = mul2(mul2(ia.se, sej), mul2(inv_r2, mul2(r6, one_m_r6)));
  const float2 coul = mul2(mul2(ia.cq, qj), fma2(inv_r2, inv_r, ia.nrc3));
  float2 gbc;
  if (kFarGb) {
    gbc = mul2(mul2(ia.gq, qj), mul2(inv_r, mul2(inv_r, inv_r)));
  } else {
    const float2 e = make_float2(exp2f(arg.x), exp2f(arg.y));
    const float2 f2 = fma2(mul2(ia.R, Rj), e, r2);
    const float2 inv_f = make_float2(rsqrtf(f2.x), rsqrtf(f2.y));
    const float2 wgt = fma2(bc(-0.25f), e, bc(1.0f));
    gbc = mul2(mul2(ia.gq, qj), mul2(wgt, mul2(inv_f, mul2(inv_f, inv_f))));
  }
  float2 c;
  if (kAllPairs) {
    c = add2(add2(ljc, coul), gbc);
  } else {
    const float2 nb = add2(ljc, coul);
    c.x = ((r2.x <= a.nb_c2) ? nb.x : 0.0f) + ((r2.x <= a.gb_c2) ? gbc.x : 0.0f);
    c.y = ((r2.y <= a.nb_c2) ? nb.y : 0.0f) + ((r2.y <= a.gb_c2) ? gbc.y : 0.0f);
  }
  c.x = (r2.x >= 1e-18f) ? c.x : 0.0f;
  c.y = (r2.y >= 1e-18f) ? c.y : 0.0f;
  return c;
}

template <bool kAllPairs, int W, int kMinBlocks, bool kPersistent>
__global__ void __launch_bounds__(W * 32, kMinBlocks) k_force(PairArgs a) {
  __shared__ __align__(128) float s_buf[2][3][kStageFloats];          // columns of pq, lj, gb
  __shared__ float s_part[W][3][kStageTiles * kTile];
  __shared__ __align__(8) uint64_t s_bar[2];
  __shared__ int s_item;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    mbar_init(&s_bar[0], 1);
    mbar_init(&s_bar[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  uint32_t g = 0;  // stages this CTA has consumed
  for (int item = next_item<kPersistent>(a, &s_item, -1); item < a.n_work;
       item = next_item<kPersistent>(a, &s_item, item)) {
  PairWork w = a.work[item];
  if (a.seg_end) w.j_end = min(w.j_end, a.seg_end[w.i_tile0]);
  if (w.j_begin >= w.j_end) continue;  // chunk culled by the cutoff (block-uniform)
  const Stager st{a.jlist, w.j_begin, w.j_end, (w.j_end - w.j_begin + kStageTiles - 1) / kStageTiles, s_bar, g};
  const float* src[3] = {a.pq, a.lj, a.gb};
  if (threadIdx.x == 0) {
    if (st.n_stages > 0) st.issue<3>(0, s_buf, src);
    if (st.n_stages > 1) st.issue<3>(1, s_buf, src);
  }

  const bool active = warp < w.n_i_tiles;
  const int it = w.i_tile0 + (active ? warp : 0);
  const int i = it * kTile + lane;
  const float px = a.pq[soa_index(i, 0)], py = a.pq[soa_index(i, 1)], pz = a.pq[soa_index(i, 2)];
  const double4 oi = a.origin[it];
  IAtom2 ia;
  {
    const float qi = a.pq[soa_index(i, 3)];
    const float Ri = a.gb[soa_index(i, 0)], iRi = a.gb[soa_index(i, 1)];
    ia.rm = bc(a.lj[soa_index(i, 0)]);
    ia.se = bc(a.lj_kj12 * a.lj[soa_index(i, 1)]);
    ia.cq = bc(-a.coul_kj * qi);
    ia.gq = bc(a.gb_pref_kj * qi);
    ia.R = bc(Ri);
    ia.nexp = bc(-0.25f * kLog2e * iRi);
    ia.nrc3 = bc(-a.inv_rc3);
  }
  int mref = a.mask_begin[it];
  const int mend = a.mask_begin[it + 1];
  double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0;

  for (int s = 0; s < st.n_stages; ++s) {
    const uint32_t gs = g + s;
    const int b = gs & 1;
    const bool ok = mbar_wait_bounded(&s_bar[b], (gs >> 1) & 1u);
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
      float* jfx = &s_part[warp][0][t * kTile];
      float* jfy = &s_part[warp][1][t * kTile];
      float* jfz = &s_part[warp][2][t * kTile];
      if (!(active && jt > it && !masked)) {
        jfx[lane] = 0.0f;
        jfy[lane] = 0.0f;
        jfz[lane] = 0.0f;
        continue;
      }
      const double4 oj = a.origin[jt];
      ia.nx = bc(-(px - static_cast<float>(oj.x - oi.x)));
      ia.ny = bc(-(py - static_cast<float>(oj.y - oi.y)));
      ia.nz = bc(-(pz - static_cast<float>(oj.z - oi.z)));
      const float* sp = &s_buf[b][0][t * 128];
      const float* sl = &s_buf[b][1][t * 128];
      const float* sg = &s_buf[b][2][t * 128];
      float2 fx = bc(0.0f), fy = bc(0.0f), fz = bc(0.0f);
OG_UNROLL(OG_FORCE_UNROLL)
      for (int k0 = 0; k0 < kTile; k0 += 4) {
        const float4 X = *reinterpret_cast<const float4*>(&sp[k0]);
        const float4 Y = *reinterpret_cast<const float4*>(&sp[32 + k0]);
        const float4 Z = *reinterpret_cast<const float4*>(&sp[64 + k0]);
        const float4 Q = *reinterpret_cast<const float4*>(&sp[96 + k0]);
        const float4 RM = *reinterpret_cast<const float4*>(&sl[k0]);
        const float4 SE = *reinterpret_cast<const float4*>(&sl[32 + k0]);
        const float4 RB = *reinterpret_cast<const float4*>(&sg[k0]);
        const float4 IR = *reinterpret_cast<const float4*>(&sg[32 + k0]);
        const Sep2 sa = sep2(make_float2(X.x, X.y), make_float2(Y.x, Y.y), make_float2(Z.x, Z.y), ia);
        const Sep2 sb = sep2(make_float2(X.z, X.w), make_float2(Y.z, Y.w), make_float2(Z.z, Z.w), ia);
        const float2 arga = gb_arg2(sa, make_float2(IR.x, IR.y), ia), argb = gb_arg2(sb, make_float2(IR.z, IR.w), ia);
        // the far GB form when every pair of the warp's group allows it
        const bool far = __all_sync(0xffffffffu, fmaxf(fmaxf(arga.x, arga.y), fmaxf(argb.x, argb.y)) < -30.0f);
        float2 ca, cb;
        if (far) {
          ca = coeff2<kAllPairs, true>(sa, arga, make_float2(Q.x, Q.y), make_float2(RM.x, RM.y),
                                       make_float2(SE.x, SE.y), make_float2(RB.x, RB.y), ia, a);
          cb = coeff2<kAllPairs, true>(sb, argb, make_float2(Q.z, Q.w), make_float2(RM.z, RM.w),
                                       make_float2(SE.z, SE.w), make_float2(RB.z, RB.w), ia, a);
        } else {
          ca = coeff2<kAllPairs, false>(sa, arga, make_float2(Q.x, Q.y), make_float2(RM.x, RM.y),
                                        make_float2(SE.x, SE.y), make_float2(RB.x, RB.y), ia, a);
          cb = coeff2<kAllPairs, false>(sb, argb, make_float2(Q.z, Q.w), make_float2(RM.z, RM.w),
                                        make_float2(SE.z, SE.w), make_float2(RB.z, RB.w), ia, a);
        }
        const float2 uxa = mul2(sa.dx, ca), uya = mul2(sa.dy, ca), uza = mul2(sa.dz, ca);
        const float2 uxb = mul2(sb.dx, cb), uyb = mul2(sb.dy, cb), uzb = mul2(sb.dz, cb);
        fx = add2(fx, add2(uxa, uxb));
        fy = add2(fy, add2(uya, uyb));
        fz = add2(fz, add2(uza, uzb));
        const float tx = reduce_scatter4(uxa.x, uxa.y, uxb.x, uxb.y, lane);
        const float ty = reduce_scatter4(uya.x, uya.y, uyb.x, uyb.y, lane);
        const float tz = reduce_scatter4(uza.x, uza.y, uzb.x, uzb.y, lane);
        if ((lane & 7) == 0) {
          jfx[k0 + (lane >> 3)] = -tx;
          jfy[k0 + (lane >> 3)] = -ty;
          jfz[k0 + (lane >> 3)] = -tz;
        }
      }
      acc0 += static_cast<double>(fx.x + fx.y);
      acc1 += static_cast<double>(fy.x + fy.y);
      acc2 += static_cast<double>(fz.x + fz.y);
    }
    __syncthreads();  // every warp is done with buffer b and has written its j partials
    if (threadIdx.x == 0 && s + 2 < st.n_stages) st.issue<3>(s + 2, s_buf, src);
    unsigned long long* dst[3] = {a.fx, a.fy, a.fz};
    flush_j<W, 3>(a, a.jlist, t0, cnt, s_part, dst, kForceScale);
  }
  g += st.n_stages;
  if (active && a.atom_valid[i]) {
    if (!(isfinite(acc0) && isfinite(acc1) && isfinite(acc2))) atomicOr(a.sys_nonfinite + a.atom_sys[i], 1);
    add_fixed(a.fx + i, acc0, kForceScale);
    add_fixed(a.fy + i, acc1, kForceScale);
    add_fixed(a.fz + i, acc2, kForceScale);
  }
  }
}

// ------------------------------------------------------ force, i pairs
// The same pair terms with two i-tiles per warp: lane l holds atom l of the
// block's tiles 2w and 2w + 1 in the two halves of every float2, so one
// FP32x2 instruction evaluates a j atom against both, and the stage's j
// columns are expanded in shared memory to (v, v) pairs to feed it.  A j
// atom's contributions from the two i atoms are summed in the lane before
// the warp reduce-scatter, which then serves eight pairs instead of four
// (in k_force the reduce-scatter is about a third of all instructions).
// Sums and their order per i atom and per j atom are as in k_force's
// structure: FP32 per j-tile and 4-atom group, FP64 across tiles, warps
// summed in a fixed order, fixed point at the end.
// Four-warp blocks at up to four per SM stage six j-tiles at a time (four in
// the other pair kernels): two block-wide barriers per stage, so a third
// fewer per pair; eight-warp blocks keep four, within the 48 KB of static
// shared memory, and so do five four-warp blocks per SM, within the SM's.
template <int W, int kMinBlocks>
constexpr int ip_stage_tiles() { return W <= 4 && kMinBlocks <= 4 ? 6 : kStageTiles; }

template <bool kAllPairs, int W, int kMinBlocks, bool kPersistent>
__global__ void __launch_bounds__(W * 32, kMinBlocks) k_force_ip(PairArgs a) {
  constexpr int kST = ip_stage_tiles<W, kMinBlocks>();
  __shared__ __align__(128) float s_buf[2][3][kST * 128];   // raw columns of pq, lj, gb (TMA)
  __shared__ __align__(16) float s_dup[3][2 * kST * 128];    // the stage's columns, each value twice
  __shared__ float s_part[W][3][kST * kTile];
  __shared__ __align__(8) uint64_t s_bar[2];
  __shared__ int s_item;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    mbar_init(&s_bar[0], 1);
    mbar_init(&s_bar[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  uint32_t g = 0;  // stages this CTA has consumed
  for (int item = next_item<kPersistent>(a, &s_item, -1); item < a.n_work;
       item = next_item<kPersistent>(a, &s_item, item)) {
  PairWork w = a.work[item];
  if (a.seg_end) w.j_end = min(w.j_end, a.seg_end[w.i_tile0]);
  if (w.j_begin >= w.j_end) continue;  // chunk culled by the cutoff (block-uniform)
  const StagerT<kST> st{a.jlist, w.j_begin, w.j_end, (w.j_end - w.j_begin + kST - 1) / kST, s_bar, g};
  const float* src[3] = {a.pq, a.lj, a.gb};
  if (threadIdx.x == 0) {
    if (st.n_stages > 0) st.issue<3>(0, s_buf, src);
    if (st.n_stages > 1) st.issue<3>(1, s_buf, src);
  }

  // tiles 2w (half x) and 2w + 1 (half y); a missing second tile repeats the
  // first, with its pairs masked out
  const bool act_a = 2 * warp < w.n_i_tiles, act_b = 2 * warp + 1 < w.n_i_tiles;
  const int it_a = w.i_tile0 + (act_a ? 2 * warp : 0);
  const int it_b = act_b ? it_a + 1 : it_a;
  const int i_a = it_a * kTile + lane, i_b = it_b * kTile + lane;
  const float2 px = make_float2(a.pq[soa_index(i_a, 0)], a.pq[soa_index(i_b, 0)]);
  const float2 py = make_float2(a.pq[soa_index(i_a, 1)], a.pq[soa_index(i_b, 1)]);
  const float2 pz = make_float2(a.pq[soa_index(i_a, 2)], a.pq[soa_index(i_b, 2)]);
  IAtom2 ia;
  {
    const float2 qi = make_float2(a.pq[soa_index(i_a, 3)], a.pq[soa_index(i_b, 3)]);
    const float2 Ri = make_float2(a.gb[soa_index(i_a, 0)], a.gb[soa_index(i_b, 0)]);
    const float2 iRi = make_float2(a.gb[soa_index(i_a, 1)], a.gb[soa_index(i_b, 1)]);
    ia.rm = make_float2(a.lj[soa_index(i_a, 0)], a.lj[soa_index(i_b, 0)]);
    ia.se = mul2(bc(a.lj_kj12), make_float2(a.lj[soa_index(i_a, 1)], a.lj[soa_index(i_b, 1)]));
    ia.cq = mul2(bc(-a.coul_kj), qi);
    ia.gq = mul2(bc(a.gb_pref_kj), qi);
    ia.R = Ri;
    ia.nexp = mul2(bc(-0.25f * kLog2e), iRi);
    ia.nrc3 = bc(-a.inv_rc3);
  }
  int mref_a = a.mask_begin[it_a], mref_b = a.mask_begin[it_b];
  const int mend_a = a.mask_begin[it_a + 1], mend_b = a.mask_begin[it_b + 1];
  double acc_ax = 0.0, acc_ay = 0.0, acc_az = 0.0, acc_bx = 0.0, acc_by = 0.0, acc_bz = 0.0;

  for (int s = 0; s < st.n_stages; ++s) {
    const uint32_t gs = g + s;
    const int b = gs & 1;
    const bool ok = mbar_wait_bounded(&s_bar[b], (gs >> 1) & 1u);
    if (__syncthreads_or(!ok)) {
      if (threadIdx.x == 0) atomicOr(a.error_flag, kStatusTimeout);
      return;
    }
    const int t0 = w.j_begin + s * kST;
    const int cnt = min(kST, w.j_end - t0);
    // expand the stage's columns: value q of an array to entries 2q, 2q + 1
#pragma unroll
    for (int c = 0; c < 3; ++c)
      for (int q = threadIdx.x; q < cnt * 128; q += W * 32) {
        const float v = s_buf[b][c][q];
        *reinterpret_cast<float2*>(&s_dup[c][2 * q]) = make_float2(v, v);
      }
    __syncthreads();  // s_dup is complete and raw buffer b is free
    if (threadIdx.x == 0 && s + 2 < st.n_stages) st.issue<3>(s + 2, s_buf, src);
    for (int t = 0; t < cnt; ++t) {
      const int jt = a.jlist[t0 + t];
      while (mref_a < mend_a && a.mask_refs[mref_a].j_tile < jt) ++mref_a;
      while (mref_b < mend_b && a.mask_refs[mref_b].j_tile < jt) ++mref_b;
      const bool va = act_a && jt > it_a && !(mref_a < mend_a && a.mask_refs[mref_a].j_tile == jt);
      const bool vb = act_b && jt > it_b && !(mref_b < mend_b && a.mask_refs[mref_b].j_tile == jt);
      float* jfx = &s_part[warp][0][t * kTile];
      float* jfy = &s_part[warp][1][t * kTile];
      float* jfz = &s_part[warp][2][t * kTile];
      if (!(va || vb)) {
        jfx[lane] = 0.0f;
        jfy[lane] = 0.0f;
        jfz[lane] = 0.0f;
        continue;
      }
      const bool both = va && vb;
      const double4 oj = a.origin[jt], oa = a.origin[it_a], ob = a.origin[it_b];
      ia.nx = make_float2(-(px.x - static_cast<float>(oj.x - oa.x)), -(px.y - static_cast<float>(oj.x - ob.x)));
      ia.ny = make_float2(-(py.x - static_cast<float>(oj.y - oa.y)), -(py.y - static_cast<float>(oj.y - ob.y)));
      ia.nz = make_float2(-(pz.x - static_cast<float>(oj.z - oa.z)), -(pz.y - static_cast<float>(oj.z - ob.z)));
      const float* dp = &s_dup[0][t * 256];
      const float* dl = &s_dup[1][t * 256];
      const float* dg = &s_dup[2][t * 256];
      float2 fx = bc(0.0f), fy = bc(0.0f), fz = bc(0.0f);
      for (int k0 = 0; k0 < kTile; k0 += 4) {
        float tjx[4], tjy[4], tjz[4];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int k2 = 2 * (k0 + 2 * h);  // two j atoms: entries k2 .. k2 + 3
          const float4 X = *reinterpret_cast<const float4*>(&dp[k2]);
          const float4 Y = *reinterpret_cast<const float4*>(&dp[64 + k2]);
          const float4 Z = *reinterpret_cast<const float4*>(&dp[128 + k2]);
          const float4 Q = *reinterpret_cast<const float4*>(&dp[192 + k2]);
          const float4 RM = *reinterpret_cast<const float4*>(&dl[k2]);
          const float4 SE = *reinterpret_cast<const float4*>(&dl[64 + k2]);
          const float4 RB = *reinterpret_cast<const float4*>(&dg[k2]);
          const float4 IR = *reinterpret_cast<const float4*>(&dg[64 + k2]);
          const Sep2 s0 = sep2(make_float2(X.x, X.y), make_float2(Y.x, Y.y), make_float2(Z.x, Z.y), ia);
          const Sep2 s1 = sep2(make_float2(X.z, X.w), make_float2(Y.z, Y.w), make_float2(Z.z, Z.w), ia);
          const float2 arg0 = gb_arg2(s0, make_float2(IR.x, IR.y), ia);
          const float2 arg1 = gb_arg2(s1, make_float2(IR.z, IR.w), ia);
          const bool far = __all_sync(0xffffffffu, fmaxf(fmaxf(arg0.x, arg0.y), fmaxf(arg1.x, arg1.y)) < -30.0f);
          float2 c0, c1;
          if (far) {
            c0 = coeff2<kAllPairs, true>(s0, arg0, make_float2(Q.x, Q.y), make_float2(RM.x, RM.y),
                                         make_float2(SE.x, SE.y), make_float2(RB.x, RB.y), ia, a);
            c1 = coeff2<kAllPairs, true>(s1, arg1, make_float2(Q.z, Q.w), make_float2(RM.z, RM.w),
                                         make_float2(SE.z, SE.w), make_float2(RB.z, RB.w), ia, a);
          } else {
            c0 = coeff2<kAllPairs, false>(s0, arg0, make_float2(Q.x, Q.y), make_float2(RM.x, RM.y),
                                          make_float2(SE.x, SE.y), make_float2(RB.x, RB.y), ia, a);
            c1 = coeff2<kAllPairs, false>(s1, arg1, make_float2(Q.z, Q.w), make_float2(RM.z, RM.w),
                                          make_float2(SE.z, SE.w), make_float2(RB.z, RB.w), ia, a);
          }
          if (!both) {  // one tile's pairs with this j-tile are near field or counted elsewhere
            c0 = make_float2(va ? c0.x : 0.0f, vb ? c0.y : 0.0f);
            c1 = make_float2(va ? c1.x : 0.0f, vb ? c1.y : 0.0f);
          }
          const float2 ux0 = mul2(s0.dx, c0), uy0 = mul2(s0.dy, c0), uz0 = mul2(s0.dz, c0);
          const float2 ux1 = mul2(s1.dx, c1), uy1 = mul2(s1.dy, c1), uz1 = mul2(s1.dz, c1);
          fx = add2(fx, add2(ux0, ux1));
          fy = add2(fy, add2(uy0, uy1));
          fz = add2(fz, add2(uz0, uz1));
          tjx[2 * h] = ux0.x + ux0.y;
          tjy[2 * h] = uy0.x + uy0.y;
          tjz[2 * h] = uz0.x + uz0.y;
          tjx[2 * h + 1] = ux1.x + ux1.y;
          tjy[2 * h + 1] = uy1.x + uy1.y;
          tjz[2 * h + 1] = uz1.x + uz1.y;
        }
        const float tx = reduce_scatter4(tjx[0], tjx[1], tjx[2], tjx[3], lane);
        const float ty = reduce_scatter4(tjy[0], tjy[1], tjy[2], tjy[3], lane);
        const float tz = reduce_scatter4(tjz[0], tjz[1], tjz[2], tjz[3], lane);
        if ((lane & 7) == 0) {
          jfx[k0 + (lane >> 3)] = -tx;
          jfy[k0 + (lane >> 3)] = -ty;
          jfz[k0 + (lane >> 3)] = -tz;
        }
      }
      acc_ax += static_cast<double>(fx.x);
      acc_ay += static_cast<double>(fy.x);
      acc_az += static_cast<double>(fz.x);
      acc_bx += static_cast<double>(fx.y);
      acc_by += static_cast<double>(fy.y);
      acc_bz += static_cast<double>(fz.y);
    }
    __syncthreads();  // every warp is done with s_dup and has written its j partials
    unsigned long long* dst[3] = {a.fx, a.fy, a.fz};
    flush_j<W, 3, kST>(a, a.jlist, t0, cnt, s_part, dst, kForceScale);
  }
  g += st.n_stages;
  if (act_a && a.atom_valid[i_a]) {
    if (!(isfinite(acc_ax) && isfinite(acc_ay) && isfinite(acc_az))) atomicOr(a.sys_nonfinite + a.atom_sys[i_a], 1);
    add_fixed(a.fx + i_a, acc_ax, kForceScale);
    add_fixed(a.fy + i_a, acc_ay, kForceScale);
    add_fixed(a.fz + i_a, acc_az, kForceScale);
  }
  if (act_b && a.atom_valid[i_b]) {
    if (!(isfinite(acc_bx) && isfinite(acc_by) && isfinite(acc_bz))) atomicOr(a.sys_nonfinite + a.atom_sys[i_b], 1);
    add_fixed(a.fx + i_b, acc_bx, kForceScale);
    add_fixed(a.fy + i_b, acc_by, kForceScale);
    add_fixed(a.fz + i_b, acc_bz, kForceScale);
  }
  }
}

}  // namespace


namespace {

// One warp per i-block; lanes test 32 j-tiles at a time against each of the
// block's i-tile spheres and append the survivors in order.
__global__ void k_cut_lists(const CutBlock* blocks, int32_t n_blocks, const int32_t* jlist_all,
                            const double4* origin, double cutoff, int32_t* jlist_out, int32_t* seg_end) {
  const int b = static_cast<int>((blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (b >= n_blocks) return;
  const CutBlock cb = blocks[b];
  int count = 0;
  for (int p0 = cb.jb; p0 < cb.je; p0 += 32) {
    const int p = p0 + lane;
    bool keep = false;
    int jt = 0;
    if (p < cb.je) {
      jt = jlist_all[p];
      const double4 oj = origin[jt];
      for (int k = 0; k < cb.n_i_tiles && !keep; ++k) {
        const double4 oi = origin[cb.i_tile0 + k];
        const double dx = oj.x - oi.x, dy = oj.y - oi.y, dz = oj.z - oi.z;
        const double lim = oi.w + oj.w + cutoff + 1e-3;
        keep = dx * dx + dy * dy + dz * dz <= lim * lim;
      }
    }
    const unsigned kept = __ballot_sync(0xffffffffu, keep);
    if (keep) jlist_out[cb.jb + count + __popc(kept & ((1u << lane) - 1u))] = jt;
    count += __popc(kept);
  }
  if (lane == 0) seg_end[cb.i_tile0] = cb.jb + count;
}

}  // namespace

void launch_cut_lists(const CutBlock* blocks, int32_t n_blocks, const int32_t* jlist_all, const double4* origin,
                      double cutoff, int32_t* jlist_out, int32_t* seg_end, cudaStream_t s) {
  if (n_blocks > 0)
    k_cut_lists<<<(n_blocks + 3) / 4, 128, 0, s>>>(blocks, n_blocks, jlist_all, origin, cutoff, jlist_out, seg_end);
}

namespace {

// A persistent launch fills the SMs with resident CTAs (at most one per item).
template <class K>
int persistent_grid(K kernel, int threads, int n_work) {
  static int n_sm = 0;
  if (n_sm == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
  }
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0);
  return std::max(1, std::min(n_work, std::max(per_sm, 1) * std::max(n_sm, 1)));
}

template <int W, int MB, bool P>
void born_variant(const PairArgs& a, cudaStream_t s) {
  auto k = k_born<W, MB, P>;
  if (P) {
    cudaMemsetAsync(a.queue, 0, sizeof(int32_t), s);
    k<<<persistent_grid(k, W * 32, a.n_work), W * 32, 0, s>>>(a);
  } else {
    k<<<a.n_work, W * 32, 0, s>>>(a);
  }
}

template <bool AP, int W, int MB, bool P>
void force_variant(const PairArgs& a, cudaStream_t s) {
  auto k = k_force<AP, W, MB, P>;
  if (P) {
    cudaMemsetAsync(a.queue, 0, sizeof(int32_t), s);
    k<<<persistent_grid(k, W * 32, a.n_work), W * 32, 0, s>>>(a);
  } else {
    k<<<a.n_work, W * 32, 0, s>>>(a);
  }
}

template <bool AP, int W, int MB, bool P>
void force_ip_variant(const PairArgs& a, cudaStream_t s) {
  auto k = k_force_ip<AP, W, MB, P>;
  if (P) {
    cudaMemsetAsync(a.queue, 0, sizeof(int32_t), s);
    k<<<persistent_grid(k, W * 32, a.n_work), W * 32, 0, s>>>(a);
  } else {
    k<<<a.n_work, W * 32, 0, s>>>(a);
  }
}

template <bool AP, bool P>
void force_shape(const PairArgs& a, int shape, cudaStream_t s) {
  switch (shape) {
    case 1: force_variant<AP, 4, 4, P>(a, s); break;
    case 2: force_variant<AP, 8, 3, P>(a, s); break;
    case 3: force_ip_variant<AP, 8, 2, P>(a, s); break;
    case 4: force_ip_variant<AP, 4, 4, P>(a, s); break;
    case 5: force_ip_variant<AP, 4, 5, P>(a, s); break;
    case 6: force_ip_variant<AP, 4, 6, P>(a, s); break;
    default: force_variant<AP, 8, 2, P>(a, s); break;
  }
}

}  // namespace

int pair_shape_tiles(int shape) {
  switch (shape) {
    case 1: return 4;
    case 3: return 16;
    default: return 8;
  }
}

void launch_born_pass(const PairArgs& a, const PairLaunch& c, cudaStream_t s) {
  if (a.n_work <= 0) return;
  if (c.persistent && !a.queue) return;
  switch (c.shape * 2 + (c.persistent ? 1 : 0)) {
    case 2: born_variant<4, 8, false>(a, s); break;
    case 3: born_variant<4, 8, true>(a, s); break;
    case 4: born_variant<8, 3, false>(a, s); break;
    case 5: born_variant<8, 3, true>(a, s); break;
    case 1: born_variant<8, 4, true>(a, s); break;
    default: born_variant<8, 4, false>(a, s); break;
  }
}

void launch_force_pass(const PairArgs& a, const PairLaunch& c, cudaStream_t s) {
  if (a.n_work <= 0) return;
  if (c.persistent && !a.queue) return;
  const bool all_pairs = a.nb_c2 == INFINITY && a.gb_c2 == INFINITY;
  if (all_pairs) {
    if (c.persistent) force_shape<true, true>(a, c.shape, s);
    else force_shape<true, false>(a, c.shape, s);
  } else {
    if (c.persistent) force_shape<false, true>(a, c.shape, s);
    else force_shape<false, false>(a, c.shape, s);
  }
}

}  // namespace ogk
