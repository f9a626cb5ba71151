// Kernels of the learned-Born-radius path (definitions in lgb.cuh).
#include <cmath>

#include "common.cuh"
#include "lgb.cuh"

namespace ogk {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr float kMu0 = 1.5f, kShell = 0.7f;
constexpr float kInv2Sigma2 = 1.0f / (2.0f * 0.7f * 0.7f);
constexpr float kCut = 12.0f;
constexpr float kPiF = 3.14159265358979f;
constexpr float kPiOverCut = kPiF / kCut;
constexpr float kLog2e = 1.4426950408889634f;
constexpr float kLn2 = 0.6931471805599453f;
constexpr float kA2 = kInv2Sigma2 * kLog2e;  // shell exponent in base 2

// Special-function-unit approximations (PTX .approx.ftz: one instruction
// each, errors of 1e-7 to 1e-6, subnormals flushed), for the descriptor
// loop only; the descriptors' tolerance is 2e-5 on log(1 + D).
__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float rsqrt_approx(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float rcp_approx(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float lg2_approx(float x) {
  float y;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float cos_approx(float x) {
  float y;
  asm("cos.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// Hawkins-Cramer-Truhlar pairwise descreening integral of atom i (offset
// radius rti) by a partner sphere of scaled radius sj at distance r, 1/r = ir
// (the standard closed form of the 1/r^4 volume integral outside atom i).
// 1/l and 1/u come from one reciprocal of l u.
__device__ __forceinline__ float hct_term(float r, float ir, float rti, float sj) {
  if (!(rti < r + sj)) return 0.0f;
  const float l = fmaxf(rti, fabsf(r - sj)), u = r + sj;
  const float q = rcp_approx(l * u);
  const float il = u * q, iu = l * q;
  float t = 0.5f * (il - iu + 0.25f * r * (iu * iu - il * il) + (0.5f * kLn2) * ir * lg2_approx(l * iu) +
                    0.25f * sj * sj * ir * (il * il - iu * iu));
  if (rti < sj - r) t += 2.0f * (rcp_approx(rti) - il);
  return t;
}

// Gaussian shells g_s = exp(-a (r - mu_s)^2), mu_s = 1.5 + 0.7 s, a = 1 /
// (2 sigma^2), by recurrence: with d = r - mu_s, g_{s+1} = g_s exp(a (2 D d -
// D^2)) and g_{s-1} = g_s exp(-a (2 D d + D^2)) (D = 0.7), and each of those
// factors changes by exp(-2 a D^2) = exp(-1) per shell (sigma = D).  Seeds at
// shells 4 and 12 run the recurrence over [0, 7] and [8, 15]: two seeds of
// four shells each side keep the error within a few 1e-6 of the shell value
// (about five times the direct evaluation's) at 6 exponentials per partner
// instead of 16, which is what bounds this kernel (the special-function
// unit).  The two runs take the same steps, so they advance together as the
// halves of packed FP32x2 values: acc[k] holds shells (k, k + 8).
__device__ __forceinline__ void add_shells(float2* acc, float r, float w) {
  constexpr float kStep = 0.36787944117144233f;  // exp(-2 a D^2) = exp(-1)
  const float da = r - (kMu0 + kShell * 4), db = r - (kMu0 + kShell * 12);
  const float2 g = make_float2(ex2_approx(-da * da * kA2), ex2_approx(-db * db * kA2));
  float2 up = make_float2(ex2_approx(kA2 * (2.0f * kShell * da - kShell * kShell)),
                          ex2_approx(kA2 * (2.0f * kShell * db - kShell * kShell)));
  float2 dn = make_float2(ex2_approx(-kA2 * (2.0f * kShell * da + kShell * kShell)),
                          ex2_approx(-kA2 * (2.0f * kShell * db + kShell * kShell)));
  const float2 w2 = make_float2(w, w), step = make_float2(kStep, kStep);
  acc[4] = __ffma2_rn(w2, g, acc[4]);
  float2 gu = g, gd = g;
#pragma unroll
  for (int s = 5; s <= 7; ++s) {
    gu = __fmul2_rn(gu, up);
    up = __fmul2_rn(up, step);
    acc[s] = __ffma2_rn(w2, gu, acc[s]);
  }
#pragma unroll
  for (int s = 3; s >= 0; --s) {
    gd = __fmul2_rn(gd, dn);
    dn = __fmul2_rn(dn, step);
    acc[s] = __ffma2_rn(w2, gd, acc[s]);
  }
}

// One block of four warps per tile of 32 i-atoms (lane = atom).  The warps
// split the partners by descriptor class, so each keeps 16 or 32 shell
// accumulators instead of 64: warps 0 and 1 take the H partners (even and
// odd partner slots -- about half of all atoms), warp 2 the C/S partners,
// warp 3 the N/P and O partners.  Each warp scans the system's tiles 32 at a
// time for bounding spheres within the cutoff, then broadcasts its partners
// of each such tile one at a time (class and slot are warp-uniform).  The
// partial shell sums and Coulomb-field integrals meet in shared memory.
// (Eight warps, splitting H four ways, measured slower: every warp repeats
// the tile scan and the partner loads.)
constexpr int kDescWarps = 4;
constexpr int kDescSlots = 5;  // one per warp, plus the second class of warp 3

__global__ void __launch_bounds__(kDescWarps * 32, 8) k_lgb_desc(LgbDescArgs a) {
  __shared__ float part[kDescSlots][16][33];  // [slot][shell][atom], padded
  __shared__ float cfa_part[kDescWarps][32];
  const int ti = blockIdx.x;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i = ti * 32 + lane;
  const bool live_i = a.atom_sys[i] >= 0;
  const int sys = a.atom_sys[ti * 32];
  const double4 oi = a.origin[ti];
  const float xi = live_i ? static_cast<float>(a.x[i] - oi.x) : 0.0f;
  const float yi = live_i ? static_cast<float>(a.y[i] - oi.y) : 0.0f;
  const float zi = live_i ? static_cast<float>(a.z[i] - oi.z) : 0.0f;
  const float rti = live_i ? static_cast<float>(a.rho_tilde[i]) : 1.0f;
  // this warp's classes (second -1 for a single class) and partner slots
  const int cls0 = warp < 2 ? 3 : (warp == 2 ? 0 : 1);
  const int cls1 = warp == 3 ? 2 : -1;
  const int stride_mask = warp < 2 ? 1 : 0;
  const int residue = warp < 2 ? warp : 0;
  float2 acc[16];  // per class, shells (k, k + 8)
#pragma unroll
  for (int k = 0; k < 16; ++k) acc[k] = make_float2(0.0f, 0.0f);
  float cfa = 0.0f;
  if (sys >= 0) {
    const int2 st = a.sys_tiles[sys];
    for (int t0 = 0; t0 < st.y; t0 += 32) {
      bool near = false;
      if (t0 + lane < st.y) {
        const double4 oj = a.origin[st.x + t0 + lane];
        const double ddx = oj.x - oi.x, ddy = oj.y - oi.y, ddz = oj.z - oi.z;
        const double lim = oi.w + oj.w + kLgbCutoff + 1e-3;
        near = ddx * ddx + ddy * ddy + ddz * ddz <= lim * lim;
      }
      unsigned tiles = __ballot_sync(kFull, near);
      while (tiles) {
        const int tj = st.x + t0 + __ffs(tiles) - 1;
        tiles &= tiles - 1;
        const int j = tj * 32 + lane;
        const bool live_j = a.atom_sys[j] >= 0;
        const int cj = live_j ? a.klass[j] : -1;
        const bool mine = (cj == cls0 || cj == cls1) && (lane & stride_mask) == residue;
        unsigned todo = __ballot_sync(kFull, mine);
        if (!todo) continue;
        const float xj = static_cast<float>(a.x[j] - oi.x);
        const float yj = static_cast<float>(a.y[j] - oi.y);
        const float zj = static_cast<float>(a.z[j] - oi.z);
        const float wj = live_j ? static_cast<float>(a.rho[j]) : 0.0f;
        const float sj = live_j ? static_cast<float>(a.srho[j]) : 0.0f;
        while (todo) {
          const int b = __ffs(todo) - 1;
          todo &= todo - 1;
          const float dx = __shfl_sync(kFull, xj, b) - xi;
          const float dy = __shfl_sync(kFull, yj, b) - yi;
          const float dz = __shfl_sync(kFull, zj, b) - zi;
          const float wb = __shfl_sync(kFull, wj, b);
          const float sb = __shfl_sync(kFull, sj, b);
          const int cb = __shfl_sync(kFull, cj, b);
          const float r2 = dx * dx + dy * dy + dz * dz;
          const bool ok = live_i && r2 < kCut * kCut && !(tj == ti && b == lane);
          if (!__any_sync(kFull, ok)) continue;  // partner out of range of the whole tile
          // r and 1/r from one reciprocal square root (r = 0 exactly for
          // the atom itself, which ok excludes)
          const float ir = rsqrt_approx(fmaxf(r2, 1e-6f));
          const float r = r2 * ir;
          const float fc = ok ? 0.5f * (cos_approx(kPiOverCut * r) + 1.0f) : 0.0f;
          const float w = wb * fc;
          if (ok) cfa += fc * hct_term(r, ir, rti, sb);
          if (cb == cls0)
            add_shells(acc, r, w);
          else
            add_shells(acc + 8, r, w);
        }
      }
    }
  }
  // partial sums -> shared memory
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    part[warp][k][lane] = acc[k].x;
    part[warp][k + 8][lane] = acc[k].y;
  }
  if (cls1 >= 0) {
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      part[4][k][lane] = acc[8 + k].x;
      part[4][k + 8][lane] = acc[8 + k].y;
    }
  }
  cfa_part[warp][lane] = cfa;
  __syncthreads();
  float4* out = reinterpret_cast<float4*>(a.xin + static_cast<int64_t>(i) * kLgbIn);
  float cfa_sum = 0.0f;
#pragma unroll
  for (int w = 0; w < kDescWarps; ++w) cfa_sum += cfa_part[w][lane];
  double rc = 1.0;
  if (live_i) {
    const double inv = fmax(1.0 / a.rho_tilde[i] - static_cast<double>(cfa_sum), 1.0 / 30.0);
    rc = 1.0 / inv;
  }
  if (warp == 0) a.r_cfa[i] = rc;
  const float4 zero = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  // warp w writes float4 chunks w, w + 4, ..., w + 16 of the atom's 20
  for (int q = warp; q < kLgbIn / 4; q += kDescWarps) {
    float4 v = zero;
    if (live_i && q < kLgbDesc / 4) {
      const int c = q >> 2, s0 = (q & 3) * 4;
      float d[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int s = s0 + e;
        d[e] = c == 3 ? part[0][s][lane] + part[1][s][lane] : part[c == 0 ? 2 : (c == 1 ? 3 : 4)][s][lane];
      }
      v = make_float4(log1pf(d[0]), log1pf(d[1]), log1pf(d[2]), log1pf(d[3]));
    } else if (live_i && q == 16) {
      const int ci = a.klass[i];
      v = make_float4(ci == 0 ? 1.0f : 0.0f, ci == 1 ? 1.0f : 0.0f, ci == 2 ? 1.0f : 0.0f, ci == 3 ? 1.0f : 0.0f);
    } else if (live_i && q == 17) {
      const double rt = a.rho_tilde[i];
      v = make_float4(static_cast<float>(rt), static_cast<float>(a.srho[i] / rt), static_cast<float>(rt / rc),
                      static_cast<float>(log(rc)));
    } else if (live_i && q == 18) {
      v = make_float4(0.0f, static_cast<float>(log(a.rho_tilde[i] / rc)), 0.0f, 0.0f);
    }
    out[q] = v;
  }
}

__global__ void k_lgb_radii(AtomArrays at, const float* h3, const float* xin, const float* params,
                            const double* r_cfa) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= at.n_padded || at.atom_sys[i] < 0) return;
  const float* w4 = params + kLgbOffW4;
  const float4* h = reinterpret_cast<const float4*>(h3 + static_cast<int64_t>(i) * kLgbHidden);
  float y = params[kLgbOffB4];
  for (int k = 0; k < kLgbNSelf; ++k) y += params[kLgbOffV + k] * xin[static_cast<int64_t>(i) * kLgbIn + kLgbDesc + k];
#pragma unroll 8
  for (int k = 0; k < kLgbHidden / 4; ++k) {
    const float4 v = h[k];
    y += w4[4 * k] * v.x + w4[4 * k + 1] * v.y + w4[4 * k + 2] * v.z + w4[4 * k + 3] * v.w;
  }
  y = fminf(fmaxf(y, -5.0f), 5.0f);
  const double r = r_cfa[i] * exp(static_cast<double>(y));
  at.born_r[i] = r;
  at.gb[soa_index(i, 0)] = static_cast<float>(r);
  at.gb[soa_index(i, 1)] = static_cast<float>(1.0 / r);
}

__global__ void k_lgb_gather(const float* x, const float* t, const int64_t* idx, int b, float* xb, float* tb) {
  const int r = blockIdx.x;
  if (r >= b) return;
  const int64_t src = idx[r];
  if (threadIdx.x < kLgbIn) xb[static_cast<int64_t>(r) * kLgbIn + threadIdx.x] = x[src * kLgbIn + threadIdx.x];
  if (threadIdx.x == 0) tb[r] = t[src];
}

__device__ __forceinline__ float silu_grad(float z) {
  const float s = 1.0f / (1.0f + __expf(-z));
  return s * (1.0f + z * (1.0f - s));
}

__global__ void k_lgb_head(const float* h3, const float* z3, const float* xb, const float* tb, const float* params,
                           int b, float* y, float* dy, float* dz3, float* loss_part) {
  __shared__ float red[256];
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  const float* w4 = params + kLgbOffW4;
  float l = 0.0f;
  if (r < b) {
    float v = params[kLgbOffB4];
    for (int k = 0; k < kLgbNSelf; ++k) v += params[kLgbOffV + k] * xb[static_cast<int64_t>(r) * kLgbIn + kLgbDesc + k];
    for (int k = 0; k < kLgbHidden; ++k) v += w4[k] * h3[static_cast<int64_t>(r) * kLgbHidden + k];
    const float d = v - tb[r];
    l = d * d;
    const float g = 2.0f * d / static_cast<float>(b);
    y[r] = v;
    dy[r] = g;
    for (int k = 0; k < kLgbHidden; ++k) {
      const int64_t o = static_cast<int64_t>(r) * kLgbHidden + k;
      dz3[o] = g * w4[k] * silu_grad(z3[o]);
    }
  }
  red[threadIdx.x] = l;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) loss_part[blockIdx.x] = red[0];
}

// Block k sums column offset + k of a row-major matrix with `stride` columns
// (weighted by dy when given; k >= cols: the column of ones) over the rows.
__global__ void k_lgb_colsum(const float* m, const float* dy, int b, int stride, int offset, int cols, float* g) {
  __shared__ float red[256];
  const int k = blockIdx.x;
  float s = 0.0f;
  for (int r = threadIdx.x; r < b; r += blockDim.x)
    s += (dy ? dy[r] : 1.0f) * (k < cols ? m[static_cast<int64_t>(r) * stride + offset + k] : 1.0f);
  red[threadIdx.x] = s;
  __syncthreads();
  for (int t = blockDim.x / 2; t > 0; t >>= 1) {
    if (threadIdx.x < t) red[threadIdx.x] += red[threadIdx.x + t];
    __syncthreads();
  }
  if (threadIdx.x == 0) g[k] = red[0];
}

__global__ void k_lgb_silu_bwd(const float* dh, const float* z, int64_t n, float* dz) {
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < n;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x)
    dz[t] = dh[t] * silu_grad(z[t]);
}

__global__ void k_lgb_adam(float* p, const float* g, float* m, float* v, int n, float lr, float c1, float c2) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const float gt = g[t];
  const float mt = 0.9f * m[t] + 0.1f * gt;
  const float vt = 0.999f * v[t] + 0.001f * gt * gt;
  m[t] = mt;
  v[t] = vt;
  p[t] -= lr * (mt / c1) / (sqrtf(vt / c2) + 1e-8f);
}

__global__ void k_lgb_force_error(const unsigned long long* fax, const unsigned long long* fay,
                                  const unsigned long long* faz, const unsigned long long* fbx,
                                  const unsigned long long* fby, const unsigned long long* fbz,
                                  const int32_t* begin, const int32_t* end, double* part) {
  __shared__ double rn[256], rd[256];
  const int s = blockIdx.x;
  double num = 0.0, den = 0.0;
  auto f = [](unsigned long long v) { return static_cast<double>(static_cast<long long>(v)) * kForceUnscale; };
  for (int i = begin[s] + threadIdx.x; i < end[s]; i += blockDim.x) {
    const double bx = f(fbx[i]), by = f(fby[i]), bz = f(fbz[i]);
    const double dx = f(fax[i]) - bx, dy = f(fay[i]) - by, dz = f(faz[i]) - bz;
    num += dx * dx + dy * dy + dz * dz;
    den += bx * bx + by * by + bz * bz;
  }
  rn[threadIdx.x] = num;
  rd[threadIdx.x] = den;
  __syncthreads();
  for (int t = blockDim.x / 2; t > 0; t >>= 1) {
    if (threadIdx.x < t) {
      rn[threadIdx.x] += rn[threadIdx.x + t];
      rd[threadIdx.x] += rd[threadIdx.x + t];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * s] = rn[0];
    part[2 * s + 1] = rd[0];
  }
}

__global__ void k_lgb_sum(const float* part, int n, float* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  float s = 0.0f;
  for (int k = 0; k < n; ++k) s += part[k];
  *out = s;
}

}  // namespace

void launch_lgb_descriptors(const LgbDescArgs& a, cudaStream_t s) {
  const int tiles = a.n_padded >> 5;
  if (tiles > 0) k_lgb_desc<<<tiles, kDescWarps * 32, 0, s>>>(a);
}

void launch_lgb_radii(const AtomArrays& at, const float* h3, const float* xin, const float* params,
                      const double* r_cfa, cudaStream_t s) {
  k_lgb_radii<<<(at.n_padded + 255) / 256, 256, 0, s>>>(at, h3, xin, params, r_cfa);
}

void launch_lgb_gather(const float* x, const float* t, const int64_t* idx, int b, float* xb, float* tb,
                       cudaStream_t s) {
  k_lgb_gather<<<b, kLgbIn, 0, s>>>(x, t, idx, b, xb, tb);
}

void launch_lgb_head(const float* h3, const float* z3, const float* xb, const float* tb, const float* params, int b,
                     float* y, float* dy, float* dz3, float* loss_part, int loss_blocks, cudaStream_t s) {
  k_lgb_head<<<loss_blocks, 256, 0, s>>>(h3, z3, xb, tb, params, b, y, dy, dz3, loss_part);
}

void launch_lgb_head_grad(const float* h3, const float* dy, int b, float* g_w4b4, cudaStream_t s) {
  k_lgb_colsum<<<kLgbHidden + 1, 256, 0, s>>>(h3, dy, b, kLgbHidden, 0, kLgbHidden, g_w4b4);
}

void launch_lgb_self_grad(const float* xb, const float* dy, int b, float* g_v, cudaStream_t s) {
  k_lgb_colsum<<<kLgbNSelf, 256, 0, s>>>(xb, dy, b, kLgbIn, kLgbDesc, kLgbNSelf, g_v);
}

void launch_lgb_colsum(const float* dz, int b, float* g, cudaStream_t s) {
  k_lgb_colsum<<<kLgbHidden, 256, 0, s>>>(dz, nullptr, b, kLgbHidden, 0, kLgbHidden, g);
}

void launch_lgb_silu_bwd(const float* dh, const float* z, int64_t n, float* dz, cudaStream_t s) {
  k_lgb_silu_bwd<<<148 * 8, 256, 0, s>>>(dh, z, n, dz);
}

void launch_lgb_adam(float* p, const float* g, float* m, float* v, int n, float lr, int t, cudaStream_t s) {
  const float c1 = 1.0f - powf(0.9f, static_cast<float>(t));
  const float c2 = 1.0f - powf(0.999f, static_cast<float>(t));
  k_lgb_adam<<<(n + 255) / 256, 256, 0, s>>>(p, g, m, v, n, lr, c1, c2);
}

void launch_lgb_sum(const float* part, int n, float* out, cudaStream_t s) { k_lgb_sum<<<1, 32, 0, s>>>(part, n, out); }

void launch_lgb_force_error(const unsigned long long* fax, const unsigned long long* fay,
                            const unsigned long long* faz, const unsigned long long* fbx,
                            const unsigned long long* fby, const unsigned long long* fbz, const int32_t* begin,
                            const int32_t* end, int n_sys, double* part, cudaStream_t s) {
  k_lgb_force_error<<<n_sys, 256, 0, s>>>(fax, fay, faz, fbx, fby, fbz, begin, end, part);
}

}  // namespace ogk
