// Gather / scatter between the padded SoA device arrays and AoS triples of
// the real atoms (definitions in state.cuh).  One thread per atom; HBM-bound
// copies (48 B per atom each way for FP64 triples).
#include "state.cuh"

namespace ogk {

namespace {

template <typename S, typename D>
__global__ void k_gather(const S* __restrict__ a, const S* __restrict__ b, const S* __restrict__ c,
                         const int32_t* __restrict__ map, int64_t n, D* __restrict__ out) {
  const int64_t g = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (g >= n) return;
  const int32_t p = map[g];
  out[3 * g] = static_cast<D>(a[p]);
  out[3 * g + 1] = static_cast<D>(b[p]);
  out[3 * g + 2] = static_cast<D>(c[p]);
}

template <typename S, typename D>
__global__ void k_scatter(const S* __restrict__ in, const int32_t* __restrict__ map, int64_t n, D* __restrict__ a,
                          D* __restrict__ b, D* __restrict__ c) {
  const int64_t g = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (g >= n) return;
  const int32_t p = map[g];
  a[p] = static_cast<D>(in[3 * g]);
  b[p] = static_cast<D>(in[3 * g + 1]);
  c[p] = static_cast<D>(in[3 * g + 2]);
}

constexpr int kThreads = 256;

inline unsigned blocks(int64_t n) { return static_cast<unsigned>((n + kThreads - 1) / kThreads); }

}  // namespace

void launch_gather_xyz(const double* a, const double* b, const double* c, const int32_t* map, int64_t n,
                       double* out, cudaStream_t s) {
  if (n > 0) k_gather<double, double><<<blocks(n), kThreads, 0, s>>>(a, b, c, map, n, out);
}

void launch_scatter_xyz(const double* in, const int32_t* map, int64_t n, double* a, double* b, double* c,
                        cudaStream_t s) {
  if (n > 0) k_scatter<double, double><<<blocks(n), kThreads, 0, s>>>(in, map, n, a, b, c);
}

// Fixed-point accumulators are two's-complement 64-bit integers held as
// unsigned long long; the conversion keeps every bit.
void launch_gather_fixed(const unsigned long long* a, const unsigned long long* b, const unsigned long long* c,
                         const int32_t* map, int64_t n, int64_t* out, cudaStream_t s) {
  if (n > 0) k_gather<unsigned long long, int64_t><<<blocks(n), kThreads, 0, s>>>(a, b, c, map, n, out);
}

void launch_scatter_fixed(const int64_t* in, const int32_t* map, int64_t n, unsigned long long* a,
                          unsigned long long* b, unsigned long long* c, cudaStream_t s) {
  if (n > 0) k_scatter<int64_t, unsigned long long><<<blocks(n), kThreads, 0, s>>>(in, map, n, a, b, c);
}

}  // namespace ogk
