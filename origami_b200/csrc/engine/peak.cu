// FP32 FMA throughput microbenchmark: the denominator of the pair kernels'
// FP32-pipe roofline (og_measure_fp32_peak).
#include <cuda_runtime.h>

#include <string>

#include "../../../include/origami_gpu.h"
#include "../host/status.h"

namespace {

constexpr int kChains = 8;
constexpr int kIters = 4096;

__global__ void k_fma_chain(float* out, float a, float b) {
  float v[kChains];
#pragma unroll
  for (int c = 0; c < kChains; ++c) v[c] = threadIdx.x * 1e-3f + c;
  for (int it = 0; it < kIters; ++it) {
#pragma unroll
    for (int c = 0; c < kChains; ++c) v[c] = fmaf(v[c], a, b);
  }
  float s = 0.0f;
#pragma unroll
  for (int c = 0; c < kChains; ++c) s += v[c];
  if (s == 12345.678f) out[threadIdx.x] = s;  // keeps the chain alive, never true in practice
}

}  // namespace

extern "C" og_status og_measure_fp32_peak(double* tflops) {
  if (!tflops) return og_fail(OG_E_BADARG, "null output");
  int dev = 0, n_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return og_fail(OG_E_CUDA, "no CUDA device");
  cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
  float* out = nullptr;
  if (cudaMalloc(&out, 1024 * sizeof(float)) != cudaSuccess) return og_fail(OG_E_NOMEM, "cudaMalloc");
  const int threads = 512, blocks = n_sm * 4;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  k_fma_chain<<<blocks, threads>>>(out, 0.999f, 1e-3f);  // warm-up
  cudaEventRecord(e0);
  const int reps = 10;
  for (int r = 0; r < reps; ++r) k_fma_chain<<<blocks, threads>>>(out, 0.999f, 1e-3f);
  cudaEventRecord(e1);
  cudaError_t err = cudaEventSynchronize(e1);
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (err != cudaSuccess) return og_fail(OG_E_CUDA, std::string("fma benchmark: ") + cudaGetErrorString(err));
  const double flops = 2.0 * kChains * static_cast<double>(kIters) * threads * blocks * reps;
  *tflops = flops / (ms * 1e-3) / 1e12;
  return OG_OK;
}
