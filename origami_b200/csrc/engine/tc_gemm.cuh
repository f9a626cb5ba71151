// BF16 tensor-core GEMM (tcgen05, FP32 accumulate) over strided FP32
// operands; see tc_gemm.cu.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace ogk {

struct TcGemmArgs {
  const float* a;
  int64_t a_sm, a_sk;   // A(m, k) = a[m * a_sm + k * a_sk]
  const float* b;
  int64_t b_sn, b_sk;   // B(n, k) = b[n * b_sn + k * b_sk]
  float* c;
  int64_t c_sm, c_sn;   // C(m, n) = c[m * c_sm + n * c_sn]
  int64_t c_split;      // set by the launcher
  int32_t m, n, k;
  int32_t k_per_split;  // set by the launcher
  const float* bias;    // optional, per n
  float* c_act;         // optional: SiLU(C) with C's strides
  int32_t* error_flag;  // kStatusTimeout on a barrier wait that ran out
};

// C = A B^T (+ bias) with `splits` K-splits; split-K needs a row-major
// contiguous C and `split_scratch` of tc_gemm_scratch_floats(m, n, splits)
// floats, else it runs unsplit.
void launch_tc_gemm(const TcGemmArgs& a, int splits, float* split_scratch, cudaStream_t s);
size_t tc_gemm_scratch_floats(int m, int n, int splits);
cudaError_t tc_gemm_prepare();

}  // namespace ogk
