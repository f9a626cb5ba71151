// Learned Born radii: the C-ABI entries of the tensor-core GEMM and of the
// network's trainer.  Training is plain minibatch Adam on the mean squared
// error of y = log(R_plainGB / R_cfa); every layer product runs on the
// tcgen05 GEMM (forward: X W^T with bias and SiLU in the epilogue; backward:
// dZ^T H and dZ W through transposed strides), the rest on small kernels.
#include <cuda_runtime.h>

#include <cmath>
#include <numeric>
#include <string>
#include <vector>

#include "../../../include/origami_gpu.h"
#include "../host/status.h"
#include "common.cuh"
#include "lgb.cuh"
#include "tc_gemm.cuh"

namespace {

og_status cuda_fail(cudaError_t e, const char* what) {
  return og_fail(OG_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define LGB_CUDA(call)                                  \
  do {                                                  \
    cudaError_t _e = (call);                            \
    if (_e != cudaSuccess) return cuda_fail(_e, #call); \
  } while (0)

// Device buffer owned by the trainer.
template <class T>
struct Buf {
  T* p = nullptr;
  ~Buf() {
    if (p) cudaFree(p);
  }
  cudaError_t alloc(size_t n) { return cudaMalloc(reinterpret_cast<void**>(&p), sizeof(T) * (n ? n : 1)); }
};

// xoshiro256++ seeded by SplitMix64 (index shuffles, initial weights).
struct Rng {
  uint64_t s[4];
  explicit Rng(uint64_t seed) {
    uint64_t z = seed;
    for (auto& v : s) {
      z += 0x9E3779B97F4A7C15ull;
      uint64_t x = z;
      x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
      x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
      v = x ^ (x >> 31);
    }
  }
  static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  uint64_t next() {
    const uint64_t r = rotl(s[0] + s[3], 23) + s[0];
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return r;
  }
  double uniform() { return static_cast<double>(next() >> 11) * (1.0 / 9007199254740992.0); }
};

using namespace ogk;

// Forward and reverse pass of one batch of B rows on the device.
struct Trainer {
  int b = 0, splits = 16;
  Buf<float> xb, tb, z1, h1, z2, h2, z3, h3, y, dy, dz3, dh, dz, g, loss_part, scratch;
  int loss_blocks = 0;
  int32_t* err = nullptr;

  cudaError_t init(int batch, int32_t* err_flag) {
    b = batch;
    err = err_flag;
    loss_blocks = (b + 255) / 256;
    cudaError_t e;
    const size_t bh = static_cast<size_t>(b) * kLgbHidden;
    for (auto* v : {&z1, &h1, &z2, &h2, &z3, &h3, &dz3, &dh, &dz})
      if ((e = v->alloc(bh)) != cudaSuccess) return e;
    if ((e = xb.alloc(static_cast<size_t>(b) * kLgbIn)) != cudaSuccess) return e;
    for (auto* v : {&tb, &y, &dy})
      if ((e = v->alloc(b)) != cudaSuccess) return e;
    if ((e = g.alloc(kLgbNParams)) != cudaSuccess) return e;
    if ((e = loss_part.alloc(loss_blocks)) != cudaSuccess) return e;
    return scratch.alloc(tc_gemm_scratch_floats(kLgbHidden, kLgbHidden, splits));
  }

  void gemm(const float* a, int64_t a_sm, int64_t a_sk, const float* bm, int64_t b_sn, int64_t b_sk, float* c,
            int64_t c_sm, int m, int n, int k, const float* bias, float* act, int nsplit, cudaStream_t s) {
    TcGemmArgs p{};
    p.a = a;
    p.a_sm = a_sm;
    p.a_sk = a_sk;
    p.b = bm;
    p.b_sn = b_sn;
    p.b_sk = b_sk;
    p.c = c;
    p.c_sm = c_sm;
    p.c_sn = 1;
    p.m = m;
    p.n = n;
    p.k = k;
    p.bias = bias;
    p.c_act = act;
    p.error_flag = err;
    launch_tc_gemm(p, nsplit, scratch.p, s);
  }

  // loss partials + gradient g of the batch already in xb / tb
  void step(const float* params, cudaStream_t s) {
    const int H = kLgbHidden;
    gemm(xb.p, kLgbIn, 1, params + kLgbOffW1, kLgbIn, 1, z1.p, H, b, H, kLgbIn, params + kLgbOffB1, h1.p, 1, s);
    gemm(h1.p, H, 1, params + kLgbOffW2, H, 1, z2.p, H, b, H, H, params + kLgbOffB2, h2.p, 1, s);
    gemm(h2.p, H, 1, params + kLgbOffW3, H, 1, z3.p, H, b, H, H, params + kLgbOffB3, h3.p, 1, s);
    launch_lgb_head(h3.p, z3.p, xb.p, tb.p, params, b, y.p, dy.p, dz3.p, loss_part.p, loss_blocks, s);
    launch_lgb_head_grad(h3.p, dy.p, b, g.p + kLgbOffW4, s);  // w4 and b4 (adjacent)
    launch_lgb_self_grad(xb.p, dy.p, b, g.p + kLgbOffV, s);
    // layer 3
    launch_lgb_colsum(dz3.p, b, g.p + kLgbOffB3, s);
    gemm(dz3.p, 1, H, h2.p, 1, H, g.p + kLgbOffW3, H, H, H, b, nullptr, nullptr, splits, s);
    gemm(dz3.p, H, 1, params + kLgbOffW3, 1, H, dh.p, H, b, H, H, nullptr, nullptr, 1, s);
    launch_lgb_silu_bwd(dh.p, z2.p, static_cast<int64_t>(b) * H, dz.p, s);
    // layer 2
    launch_lgb_colsum(dz.p, b, g.p + kLgbOffB2, s);
    gemm(dz.p, 1, H, h1.p, 1, H, g.p + kLgbOffW2, H, H, H, b, nullptr, nullptr, splits, s);
    gemm(dz.p, H, 1, params + kLgbOffW2, 1, H, dh.p, H, b, H, H, nullptr, nullptr, 1, s);
    launch_lgb_silu_bwd(dh.p, z1.p, static_cast<int64_t>(b) * H, dz3.p, s);  // dz1 into dz3's storage
    // layer 1
    launch_lgb_colsum(dz3.p, b, g.p + kLgbOffB1, s);
    gemm(dz3.p, 1, H, xb.p, 1, kLgbIn, g.p + kLgbOffW1, kLgbIn, H, kLgbIn, b, nullptr, nullptr, splits, s);
  }
};

// Least-squares fit of the output's linear path, t ~ b4 + v . x[64..80), by
// FP64 normal equations with a small ridge term (constant self features make
// them singular otherwise), solved by Cholesky.
void fit_linear_path(const float* x, const float* t, int64_t n, float* params) {
  constexpr int d = kLgbNSelf + 1;  // v and the bias
  double a[d][d] = {}, rhs[d] = {};
  double f[d];
  for (int64_t r = 0; r < n; ++r) {
    for (int k = 0; k < kLgbNSelf; ++k) f[k] = x[r * kLgbIn + kLgbDesc + k];
    f[kLgbNSelf] = 1.0;
    for (int p = 0; p < d; ++p) {
      rhs[p] += f[p] * t[r];
      for (int q = 0; q <= p; ++q) a[p][q] += f[p] * f[q];
    }
  }
  double tr = 0.0;
  for (int p = 0; p < d; ++p) tr += a[p][p];
  for (int p = 0; p < d; ++p) {
    a[p][p] += 1e-10 * tr / d + 1e-30;
    for (int q = p + 1; q < d; ++q) a[p][q] = a[q][p];
  }
  // Cholesky a = L L^T in place (lower), then two triangular solves
  for (int j = 0; j < d; ++j) {
    double s = a[j][j];
    for (int k = 0; k < j; ++k) s -= a[j][k] * a[j][k];
    a[j][j] = std::sqrt(std::max(s, 1e-300));
    for (int i = j + 1; i < d; ++i) {
      double u = a[i][j];
      for (int k = 0; k < j; ++k) u -= a[i][k] * a[j][k];
      a[i][j] = u / a[j][j];
    }
  }
  double z[d], w[d];
  for (int i = 0; i < d; ++i) {
    double u = rhs[i];
    for (int k = 0; k < i; ++k) u -= a[i][k] * z[k];
    z[i] = u / a[i][i];
  }
  for (int i = d - 1; i >= 0; --i) {
    double u = z[i];
    for (int k = i + 1; k < d; ++k) u -= a[k][i] * w[k];
    w[i] = u / a[i][i];
  }
  for (int k = 0; k < kLgbNSelf; ++k) params[kLgbOffV + k] = static_cast<float>(w[k]);
  params[kLgbOffB4] = static_cast<float>(w[kLgbNSelf]);
}

og_status check_samples(const float* x, const float* t, int64_t n) {
  if (!x || !t) return og_fail(OG_E_BADARG, "null samples");
  if (n <= 0) return og_fail(OG_E_BADARG, "no samples");
  return OG_OK;
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

og_status og_lgb_init_params(uint64_t seed, float* params) {
  if (!params) return og_fail(OG_E_BADARG, "null output");
  Rng rng(seed);
  auto fill = [&](int off, int count, int fan_in) {
    const double lim = 1.0 / std::sqrt(static_cast<double>(fan_in));
    for (int k = 0; k < count; ++k) params[off + k] = static_cast<float>((2.0 * rng.uniform() - 1.0) * lim);
  };
  const int H = kLgbHidden;
  fill(kLgbOffW1, H * kLgbIn, kLgbIn);
  fill(kLgbOffW2, H * H, H);
  fill(kLgbOffW3, H * H, H);
  for (int k = 0; k < H; ++k) params[kLgbOffW4 + k] = 0.0f;  // the network starts at output 0
  for (int off : {kLgbOffB1, kLgbOffB2, kLgbOffB3})
    for (int k = 0; k < H; ++k) params[off + k] = 0.0f;
  params[kLgbOffB4] = 0.0f;
  for (int k = 0; k < kLgbNSelf; ++k) params[kLgbOffV + k] = 0.0f;
  return OG_OK;
}

og_status og_lgb_loss_and_gradient(const float* x, const float* target, int64_t n, const float* params, double* loss,
                                   float* grad) {
  og_status st = check_samples(x, target, n);
  if (st != OG_OK) return st;
  if (!params) return og_fail(OG_E_BADARG, "null parameters");
  if (n > (1 << 20)) return og_fail(OG_E_BADARG, "at most 2^20 rows in one gradient");
  LGB_CUDA(tc_gemm_prepare());
  const int b = static_cast<int>(n);
  Buf<int32_t> err;
  Buf<float> p, sum;
  LGB_CUDA(err.alloc(1));
  LGB_CUDA(p.alloc(kLgbNParams));
  LGB_CUDA(sum.alloc(1));
  Trainer tr;
  LGB_CUDA(tr.init(b, err.p));
  cudaStream_t s = nullptr;
  LGB_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int32_t), s));
  LGB_CUDA(cudaMemcpyAsync(p.p, params, sizeof(float) * kLgbNParams, cudaMemcpyHostToDevice, s));
  LGB_CUDA(cudaMemcpyAsync(tr.xb.p, x, sizeof(float) * kLgbIn * b, cudaMemcpyHostToDevice, s));
  LGB_CUDA(cudaMemcpyAsync(tr.tb.p, target, sizeof(float) * b, cudaMemcpyHostToDevice, s));
  tr.step(p.p, s);
  launch_lgb_sum(tr.loss_part.p, tr.loss_blocks, sum.p, s);
  LGB_CUDA(cudaGetLastError());
  float l = 0.0f;
  int32_t flag = 0;
  LGB_CUDA(cudaMemcpyAsync(&l, sum.p, sizeof(float), cudaMemcpyDeviceToHost, s));
  LGB_CUDA(cudaMemcpyAsync(&flag, err.p, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  if (grad) LGB_CUDA(cudaMemcpyAsync(grad, tr.g.p, sizeof(float) * kLgbNParams, cudaMemcpyDeviceToHost, s));
  LGB_CUDA(cudaStreamSynchronize(s));
  if (flag) return og_fail(OG_E_TIMEOUT, "tensor-core GEMM barrier wait timed out");
  if (loss) *loss = static_cast<double>(l) / b;
  return OG_OK;
}

og_status og_lgb_train(const float* x, const float* target, int64_t n, int32_t steps, int32_t batch, double lr,
                       uint64_t seed, float* params, float* loss_per_step) {
  og_status st = check_samples(x, target, n);
  if (st != OG_OK) return st;
  if (!params) return og_fail(OG_E_BADARG, "null parameters");
  if (steps < 0 || batch <= 0 || batch > (1 << 20) || !(lr > 0.0)) return og_fail(OG_E_BADARG, "bad training options");
  LGB_CUDA(tc_gemm_prepare());
  cudaStream_t s = nullptr;
  const int b = static_cast<int>(std::min<int64_t>(batch, n));
  Buf<int32_t> err;
  Buf<float> p, m, v, xd, td, hist;
  Buf<int64_t> perm;
  LGB_CUDA(err.alloc(1));
  for (auto* q : {&p, &m, &v}) LGB_CUDA(q->alloc(kLgbNParams));
  LGB_CUDA(xd.alloc(static_cast<size_t>(n) * kLgbIn));
  LGB_CUDA(td.alloc(static_cast<size_t>(n)));
  LGB_CUDA(perm.alloc(static_cast<size_t>(n)));
  LGB_CUDA(hist.alloc(static_cast<size_t>(steps) + 1));
  Trainer tr;
  LGB_CUDA(tr.init(b, err.p));
  LGB_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int32_t), s));
  LGB_CUDA(cudaMemsetAsync(m.p, 0, sizeof(float) * kLgbNParams, s));
  LGB_CUDA(cudaMemsetAsync(v.p, 0, sizeof(float) * kLgbNParams, s));
  fit_linear_path(x, target, n, params);
  LGB_CUDA(cudaMemcpyAsync(p.p, params, sizeof(float) * kLgbNParams, cudaMemcpyHostToDevice, s));
  LGB_CUDA(cudaMemcpyAsync(xd.p, x, sizeof(float) * kLgbIn * n, cudaMemcpyHostToDevice, s));
  LGB_CUDA(cudaMemcpyAsync(td.p, target, sizeof(float) * n, cudaMemcpyHostToDevice, s));
  Rng rng(seed);
  std::vector<int64_t> order(static_cast<size_t>(n));
  std::iota(order.begin(), order.end(), 0);
  int64_t cursor = n;  // forces a shuffle before the first batch
  for (int t = 1; t <= steps; ++t) {
    if (cursor + b > n) {
      for (int64_t k = n - 1; k > 0; --k) std::swap(order[k], order[static_cast<int64_t>(rng.next() % (k + 1))]);
      LGB_CUDA(cudaMemcpyAsync(perm.p, order.data(), sizeof(int64_t) * n, cudaMemcpyHostToDevice, s));
      LGB_CUDA(cudaStreamSynchronize(s));  // `order` is rewritten by the next shuffle
      cursor = 0;
    }
    launch_lgb_gather(xd.p, td.p, perm.p + cursor, b, tr.xb.p, tr.tb.p, s);
    cursor += b;
    tr.step(p.p, s);
    launch_lgb_sum(tr.loss_part.p, tr.loss_blocks, hist.p + t - 1, s);
    // cosine decay of the step size over the run
    const double lr_t = lr * 0.5 * (1.0 + std::cos(M_PI * (t - 1) / std::max(steps, 1)));
    launch_lgb_adam(p.p, tr.g.p, m.p, v.p, kLgbNParams, static_cast<float>(lr_t), t, s);
  }
  LGB_CUDA(cudaGetLastError());
  std::vector<float> h(static_cast<size_t>(steps));
  int32_t flag = 0;
  LGB_CUDA(cudaMemcpyAsync(params, p.p, sizeof(float) * kLgbNParams, cudaMemcpyDeviceToHost, s));
  if (steps > 0) LGB_CUDA(cudaMemcpyAsync(h.data(), hist.p, sizeof(float) * steps, cudaMemcpyDeviceToHost, s));
  LGB_CUDA(cudaMemcpyAsync(&flag, err.p, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  LGB_CUDA(cudaStreamSynchronize(s));
  if (flag) return og_fail(OG_E_TIMEOUT, "tensor-core GEMM barrier wait timed out");
  if (loss_per_step)
    for (int t = 0; t < steps; ++t) loss_per_step[t] = h[t] / static_cast<float>(b);
  return OG_OK;
}

}  // extern "C"
