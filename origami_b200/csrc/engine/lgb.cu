// Learned Born radii: the C-ABI entries around the tensor-core GEMM.
#include <cuda_runtime.h>

#include <string>

#include "../../../include/origami_gpu.h"
#include "../host/status.h"
#include "common.cuh"
#include "tc_gemm.cuh"

namespace {

og_status cuda_fail(cudaError_t e, const char* what) {
  return og_fail(OG_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace

extern "C" {

og_status og_tc_gemm(const float* a, int64_t a_sm, int64_t a_sk, const float* b, int64_t b_sn, int64_t b_sk,
                     float* c, int64_t c_sm, int64_t c_sn, int32_t m, int32_t n, int32_t k, const float* bias,
                     float* c_act, int32_t splits, void* cuda_stream) {
  if (!a || !b || !c) return og_fail(OG_E_BADARG, "null operand");
  if (m <= 0 || n <= 0 || k <= 0) return og_fail(OG_E_BADARG, "m, n and k must be positive");
  cudaError_t e = ogk::tc_gemm_prepare();
  if (e != cudaSuccess) return cuda_fail(e, "tc_gemm_prepare");
  cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
  int32_t* err = nullptr;
  float* scratch = nullptr;
  if ((e = cudaMalloc(&err, sizeof(int32_t))) != cudaSuccess) return cuda_fail(e, "cudaMalloc");
  if (splits > 1 && c_sm == n && c_sn == 1) {
    e = cudaMalloc(&scratch, sizeof(float) * ogk::tc_gemm_scratch_floats(m, n, splits));
    if (e != cudaSuccess) {
      cudaFree(err);
      return cuda_fail(e, "cudaMalloc");
    }
  }
  cudaMemsetAsync(err, 0, sizeof(int32_t), s);
  ogk::TcGemmArgs p{};
  p.a = a;
  p.a_sm = a_sm;
  p.a_sk = a_sk;
  p.b = b;
  p.b_sn = b_sn;
  p.b_sk = b_sk;
  p.c = c;
  p.c_sm = c_sm;
  p.c_sn = c_sn;
  p.m = m;
  p.n = n;
  p.k = k;
  p.bias = bias;
  p.c_act = c_act;
  p.error_flag = err;
  ogk::launch_tc_gemm(p, splits, scratch, s);
  e = cudaGetLastError();
  int32_t flag = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&flag, err, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(err);
  if (scratch) cudaFree(scratch);
  if (e != cudaSuccess) return cuda_fail(e, "tensor-core GEMM");
  if (flag) return og_fail(OG_E_TIMEOUT, "tensor-core GEMM barrier wait timed out");
  return OG_OK;
}

}  // extern "C"
