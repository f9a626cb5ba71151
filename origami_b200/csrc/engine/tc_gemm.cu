// BF16 tensor-core GEMM with FP32 operands in global memory:
//   C[m, n] = sum_k A(m, k) B(n, k)   (+ bias[n], optional SiLU copy)
// A(m, k) = a[m * a_sm + k * a_sk], B(n, k) = b[n * b_sn + k * b_sk], so a
// transposed operand is just a different pair of strides.  One CTA (four
// warps) owns a 128 x 128 output tile; K is staged in chunks of 64 as BF16
// core matrices (tc.cuh), each chunk four tcgen05 MMAs into one TMEM
// accumulator, and the epilogue reads TMEM row by row (thread = row).
// blockIdx.z splits K; split z writes its partial to c + z * c_split and
// launch_tc_gemm sums the partials in a fixed order.
#include <cuda_bf16.h>

#include <algorithm>

#include "common.cuh"
#include "tc.cuh"
#include "tc_gemm.cuh"

namespace ogk {

namespace {

constexpr int kBM = 128, kBN = 128, kBK = 64;
constexpr uint32_t kTmemCols = 128;
// Dynamic shared memory per CTA: enough that at most four CTAs share an SM,
// so their TMEM (128 columns each) always fits the 512 columns at once and
// an allocation never waits for another CTA.
constexpr size_t kGemmSmem = 56 * 1024;

struct GemmSmem {
  uint8_t a[kBM * kBK * 2];
  uint8_t b[kBN * kBK * 2];
  uint64_t bar;
  uint32_t tmem;
};
static_assert(sizeof(GemmSmem) + 1024 <= kGemmSmem, "GEMM shared memory");

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }

__global__ void __launch_bounds__(128, 1) k_tc_gemm(TcGemmArgs p) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  // 1024-byte alignment of the operand tiles
  GemmSmem& s = *reinterpret_cast<GemmSmem*>(smem_raw + ((1024 - (smem_addr(smem_raw) & 1023)) & 1023));
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * kBN, split = blockIdx.z;
  const int k_begin = split * p.k_per_split;
  const int k_end = min(p.k, k_begin + p.k_per_split);

  if (warp == 0) tc::tmem_alloc(&s.tmem, kTmemCols);
  if (tid == 0) {
    mbar_init(&s.bar, 1);
    fence_mbar_init();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = s.tmem;
  const uint32_t idesc = tc::idesc_bf16_f32(kBM, kBN);
  constexpr uint32_t kLboA = (kBM / 8) * 128, kLboB = (kBN / 8) * 128;

  uint32_t phase = 0;
  bool ok = true;
  int chunks = 0;
  for (int k0 = k_begin; k0 < k_end && ok; k0 += kBK, ++chunks) {
    // stage: thread r converts row r of the A and B chunks
    const int gm = m0 + tid, gn = n0 + tid;
    for (int kc = 0; kc < kBK; kc += 8) {
      __align__(16) __nv_bfloat16 va[8], vb[8];
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        const int gk = k0 + kc + e;
        const bool kin = gk < k_end;
        const float x = (kin && gm < p.m) ? p.a[gm * p.a_sm + gk * p.a_sk] : 0.0f;
        const float y = (kin && gn < p.n) ? p.b[gn * p.b_sn + gk * p.b_sk] : 0.0f;
        va[e] = __float2bfloat16_rn(x);
        vb[e] = __float2bfloat16_rn(y);
      }
      *reinterpret_cast<uint4*>(s.a + tc::core_offset(tid, kc, kBM)) = *reinterpret_cast<const uint4*>(va);
      *reinterpret_cast<uint4*>(s.b + tc::core_offset(tid, kc, kBN)) = *reinterpret_cast<const uint4*>(vb);
    }
    tc::fence_smem_to_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (tid == 0) {
#pragma unroll
      for (int j = 0; j < kBK / 16; ++j) {
        const uint64_t ad = tc::smem_desc(s.a + j * 2 * kLboA, kLboA, 128);
        const uint64_t bd = tc::smem_desc(s.b + j * 2 * kLboB, kLboB, 128);
        tc::mma_bf16(tmem, ad, bd, idesc, chunks > 0 || j > 0);
      }
      tc::mma_commit(&s.bar);
    }
    // the chunk's MMAs must finish before its tiles are overwritten; after a
    // wait that ran out, wait once more (bounded) so the accumulator is not
    // freed under MMAs still in flight, then report the timeout
    if (!mbar_wait_bounded(&s.bar, phase)) {
      ok = false;
      mbar_wait_bounded(&s.bar, phase);
    }
    phase ^= 1u;
    tc::fence_after_sync();
    ok = __syncthreads_and(ok);
  }

  if (!ok) {
    if (tid == 0 && p.error_flag) atomicOr(p.error_flag, kStatusTimeout);
  } else {
    const int row = m0 + warp * 32 + lane;
    float* c = p.c + static_cast<int64_t>(split) * p.c_split;
    const bool final = gridDim.z == 1;
    for (int c0 = 0; c0 < kBN; c0 += 32) {
      float v[32];
      if (chunks > 0) {
        tc::tmem_ld32(tmem + (static_cast<uint32_t>(warp * 32) << 16) + static_cast<uint32_t>(c0), v);
      } else {
#pragma unroll
        for (int e = 0; e < 32; ++e) v[e] = 0.0f;
      }
      if (row < p.m) {
#pragma unroll
        for (int e = 0; e < 32; ++e) {
          const int n = n0 + c0 + e;
          if (n >= p.n) continue;
          float val = v[e];
          if (final && p.bias) val += p.bias[n];
          c[row * p.c_sm + n * p.c_sn] = val;
          if (final && p.c_act) p.c_act[row * p.c_sm + n * p.c_sn] = silu(val);
        }
      }
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, kTmemCols);
}

// Fixed-order sum of split-K partials (+ bias, SiLU copy).
__global__ void k_tc_reduce(TcGemmArgs p, int splits, float* out) {
  const int64_t total = static_cast<int64_t>(p.m) * p.n;
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int m = static_cast<int>(t / p.n), n = static_cast<int>(t % p.n);
    const int64_t off = m * p.c_sm + n * p.c_sn;
    float acc = 0.0f;
    for (int z = 0; z < splits; ++z) acc += p.c[z * p.c_split + off];
    if (p.bias) acc += p.bias[n];
    out[off] = acc;
    if (p.c_act) p.c_act[off] = silu(acc);
  }
}

}  // namespace

cudaError_t tc_gemm_prepare() {
  return cudaFuncSetAttribute(k_tc_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kGemmSmem));
}

void launch_tc_gemm(const TcGemmArgs& args, int splits, float* split_scratch, cudaStream_t s) {
  if (args.m <= 0 || args.n <= 0) return;
  TcGemmArgs p = args;
  splits = max(1, splits);
  // split-K only into a contiguous row-major C (the reduction's layout)
  if (!split_scratch || p.c_sm != p.n || p.c_sn != 1) splits = 1;
  const int chunks = (p.k + kBK - 1) / kBK;
  splits = min(splits, max(1, chunks));
  p.k_per_split = ((chunks + splits - 1) / splits) * kBK;
  splits = (p.k + p.k_per_split - 1) / p.k_per_split;
  if (splits < 1) splits = 1;
  dim3 grid((p.m + kBM - 1) / kBM, (p.n + kBN - 1) / kBN, splits);
  if (splits == 1) {
    p.c_split = 0;
    k_tc_gemm<<<grid, 128, kGemmSmem, s>>>(p);
    return;
  }
  // partials in the scratch (splits x m x n, row-major), then the reduction
  TcGemmArgs q = p;
  q.c = split_scratch;
  q.c_sm = p.n;
  q.c_sn = 1;
  q.c_split = static_cast<int64_t>(p.m) * p.n;
  q.bias = nullptr;
  q.c_act = nullptr;
  k_tc_gemm<<<grid, 128, kGemmSmem, s>>>(q);
  TcGemmArgs r = q;
  r.bias = p.bias;
  r.c_act = p.c_act;
  const int64_t total = static_cast<int64_t>(p.m) * p.n;
  const int64_t want = (total + 255) / 256;
  const int blocks = static_cast<int>(want < 148 * 16 ? want : 148 * 16);
  k_tc_reduce<<<blocks, 256, 0, s>>>(r, splits, p.c);
}

size_t tc_gemm_scratch_floats(int m, int n, int splits) { return static_cast<size_t>(max(1, splits)) * m * n; }

}  // namespace ogk
