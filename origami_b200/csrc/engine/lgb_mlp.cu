// Fused inference of the learned-Born-radius network: one persistent CTA per
// SM keeps W1..W3 in shared memory as BF16 core matrices (tc.cuh) and walks
// 128-atom tiles; per tile the three hidden layers are tcgen05 MMAs into one
// TMEM accumulator, each epilogue (bias, SiLU, BF16) writing the next
// layer's operand back into shared memory -- eight warps, two per TMEM lane
// quarter, each taking half of the 128 columns -- and the last epilogue finishes
// the head (w4 . h3 + b4 + v . xself) and the radius R = R_cfa exp(y) in
// registers.  Global traffic per atom: its 80 inputs in, its radius out.
// Rounding points are those of the unfused path (BF16 operands, FP32
// accumulate, FP32 bias / SiLU / head).
#include <cuda_bf16.h>

#include "common.cuh"
#include "lgb.cuh"
#include "tc.cuh"

namespace ogk {

namespace {

constexpr int kRows = 128;
constexpr int kH = kLgbHidden;
constexpr uint32_t kTmemCols = 128;
constexpr uint32_t kLbo = (kRows / 8) * 128;  // 128 rows -> 16 row groups of 128 B

struct MlpSmem {
  uint8_t w1[kH * kLgbIn * 2];
  uint8_t w2[kH * kH * 2];
  uint8_t w3[kH * kH * 2];
  uint8_t act[kRows * kH * 2];
  float b1[kH], b2[kH], b3[kH], w4[kH];
  float v[kLgbNSelf];
  float part[kRows];  // the second column half's share of the head
  uint64_t bar;
  uint32_t tmem;
};
constexpr size_t kMlpSmem = sizeof(MlpSmem) + 1024;

__device__ __forceinline__ float silu(float z) { return __fdividef(z, 1.0f + __expf(-z)); }

// W (out x in, FP32 row-major) -> BF16 core matrices with `in` along K.
__device__ void stage_weights(const float* w, int in, uint8_t* dst) {
  for (int idx = threadIdx.x; idx < kH * (in / 8); idx += blockDim.x) {
    const int r = idx / (in / 8), kc = (idx % (in / 8)) * 8;
    __align__(16) __nv_bfloat16 v[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) v[e] = __float2bfloat16_rn(w[r * in + kc + e]);
    *reinterpret_cast<uint4*>(dst + tc::core_offset(r, kc, kH)) = *reinterpret_cast<const uint4*>(v);
  }
}

// One layer: D = act[:, 0:k] W^T into TMEM, k = 80 or 128.
__device__ __forceinline__ void issue_layer(const MlpSmem& s, const uint8_t* w, int k, uint32_t tmem,
                                            uint32_t idesc) {
  for (int j = 0; j < k / 16; ++j) {
    const uint64_t ad = tc::smem_desc(s.act + j * 2 * kLbo, kLbo, 128);
    const uint64_t bd = tc::smem_desc(w + j * 2 * kLbo, kLbo, 128);
    tc::mma_bf16(tmem, ad, bd, idesc, j > 0);
  }
}

// Epilogue of a hidden layer for this thread's row and column half: h =
// SiLU(acc + b) as BF16 into act (the next layer's operand); with `head`,
// the head dot over those columns instead.
__device__ __forceinline__ float epilogue(MlpSmem& s, uint32_t taddr, const float* bias, int row, int half,
                                          bool head) {
  float y = 0.0f;
  for (int c0 = half * (kH / 2); c0 < (half + 1) * (kH / 2); c0 += 32) {
    float v[32];
    tc::tmem_ld32(taddr + static_cast<uint32_t>(c0), v);
    if (head) {
#pragma unroll
      for (int e = 0; e < 32; ++e) y += s.w4[c0 + e] * silu(v[e] + bias[c0 + e]);
    } else {
#pragma unroll
      for (int g = 0; g < 32; g += 8) {
        __align__(16) __nv_bfloat16 h[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) h[e] = __float2bfloat16_rn(silu(v[g + e] + bias[c0 + g + e]));
        *reinterpret_cast<uint4*>(s.act + tc::core_offset(row, c0 + g, kRows)) = *reinterpret_cast<const uint4*>(h);
      }
    }
  }
  return y;
}

__global__ void __launch_bounds__(256, 1) k_lgb_mlp_radii(AtomArrays at, const float* xin, const float* params,
                                                          const double* r_cfa, int32_t* error_flag) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  MlpSmem& s = *reinterpret_cast<MlpSmem*>(smem_raw + ((1024 - (smem_addr(smem_raw) & 1023)) & 1023));
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int quarter = warp & 3, half = warp >> 2;
  const int row = quarter * 32 + lane;  // the tile row (TMEM lane) this thread serves

  if (warp == 0) tc::tmem_alloc(&s.tmem, kTmemCols);
  if (tid == 0) {
    mbar_init(&s.bar, 1);
    fence_mbar_init();
  }
  stage_weights(params + kLgbOffW1, kLgbIn, s.w1);
  stage_weights(params + kLgbOffW2, kH, s.w2);
  stage_weights(params + kLgbOffW3, kH, s.w3);
  for (int k = tid; k < kH; k += blockDim.x) {
    s.b1[k] = params[kLgbOffB1 + k];
    s.b2[k] = params[kLgbOffB2 + k];
    s.b3[k] = params[kLgbOffB3 + k];
    s.w4[k] = params[kLgbOffW4 + k];
  }
  if (tid < kLgbNSelf) s.v[tid] = params[kLgbOffV + tid];
  const float b4 = params[kLgbOffB4];
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = s.tmem;
  const uint32_t taddr = tmem + (static_cast<uint32_t>(quarter * 32) << 16);
  const uint32_t idesc = tc::idesc_bf16_f32(kRows, kH);

  uint32_t phase = 0;
  bool ok = true;
  const int n_tiles = (at.n_padded + kRows - 1) / kRows;
  for (int tile = blockIdx.x; tile < n_tiles && ok; tile += gridDim.x) {
    const int i = tile * kRows + row;  // this thread's atom
    const bool live = i < at.n_padded && at.atom_sys[i] >= 0;
    // stage this thread's half of the input row (40 of 80 values) as BF16;
    // the second half holds the self features the head also reads
    constexpr int kHalfIn = kLgbIn / 2;
    const float* xr = xin + static_cast<int64_t>(i) * kLgbIn + half * kHalfIn;
    float4 xv[kHalfIn / 4];
#pragma unroll
    for (int q = 0; q < kHalfIn / 4; ++q)
      xv[q] = i < at.n_padded ? reinterpret_cast<const float4*>(xr)[q] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
#pragma unroll
    for (int kc = 0; kc < kHalfIn; kc += 8) {
      const float4 a = xv[kc / 4], b = xv[kc / 4 + 1];
      __align__(16) __nv_bfloat16 h[8];
      h[0] = __float2bfloat16_rn(a.x);
      h[1] = __float2bfloat16_rn(a.y);
      h[2] = __float2bfloat16_rn(a.z);
      h[3] = __float2bfloat16_rn(a.w);
      h[4] = __float2bfloat16_rn(b.x);
      h[5] = __float2bfloat16_rn(b.y);
      h[6] = __float2bfloat16_rn(b.z);
      h[7] = __float2bfloat16_rn(b.w);
      *reinterpret_cast<uint4*>(s.act + tc::core_offset(row, half * kHalfIn + kc, kRows)) =
          *reinterpret_cast<const uint4*>(h);
    }
    float y = half == 0 ? b4 : 0.0f;
    for (int layer = 0; layer < 3 && ok; ++layer) {
      tc::fence_smem_to_async();
      tc::fence_before_sync();
      __syncthreads();
      tc::fence_after_sync();
      if (tid == 0) {
        issue_layer(s, layer == 0 ? s.w1 : (layer == 1 ? s.w2 : s.w3), layer == 0 ? kLgbIn : kH, tmem, idesc);
        tc::mma_commit(&s.bar);
      }
      if (!mbar_wait_bounded(&s.bar, phase)) {
        ok = false;
        mbar_wait_bounded(&s.bar, phase);  // let MMAs in flight finish before TMEM is freed
      }
      phase ^= 1u;
      tc::fence_after_sync();
      ok = __syncthreads_and(ok);
      if (!ok) break;
      const float* bias = layer == 0 ? s.b1 : (layer == 1 ? s.b2 : s.b3);
      y += epilogue(s, taddr, bias, row, half, layer == 2);
    }
    if (!ok) break;
    // the second half adds the linear path (its inputs hold the self
    // features) and hands its share to the first half
    if (half == 1) {
#pragma unroll
      for (int k = 0; k < kLgbNSelf; k += 4) {
        const float4 f = xv[(kLgbDesc - kHalfIn + k) / 4];
        y += s.v[k] * f.x + s.v[k + 1] * f.y + s.v[k + 2] * f.z + s.v[k + 3] * f.w;
      }
      s.part[row] = y;
    }
    __syncthreads();
    if (half == 0 && live) {
      y += s.part[row];
      y = fminf(fmaxf(y, -5.0f), 5.0f);
      const double r = r_cfa[i] * exp(static_cast<double>(y));
      at.born_r[i] = r;
      at.gb[soa_index(i, 0)] = static_cast<float>(r);
      at.gb[soa_index(i, 1)] = static_cast<float>(1.0 / r);
    }
  }
  if (!ok && tid == 0 && error_flag) atomicOr(error_flag, kStatusTimeout);
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, kTmemCols);
  (void)lane;
}

}  // namespace

cudaError_t lgb_mlp_prepare() {
  return cudaFuncSetAttribute(k_lgb_mlp_radii, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              static_cast<int>(kMlpSmem));
}

void launch_lgb_mlp_radii(const AtomArrays& at, const float* xin, const float* params, const double* r_cfa,
                          int32_t* error_flag, int n_sm, cudaStream_t s) {
  const int tiles = (at.n_padded + kRows - 1) / kRows;
  const int grid = tiles < n_sm ? tiles : n_sm;
  if (grid <= 0) return;
  k_lgb_mlp_radii<<<grid, 256, kMlpSmem, s>>>(at, xin, params, r_cfa, error_flag);
}

}  // namespace ogk
