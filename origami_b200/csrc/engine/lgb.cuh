// Learned Born radii: per-atom environment descriptors, a Coulomb-field
// baseline radius and the kernels around the 64-128-128-128-1 SiLU network
// (whose three hidden layers run on the tensor-core GEMM of tc_gemm.cuh).
//
// Descriptor of atom i (64 values, class-major): for each partner j != i of
// the same system with r = |r_ij| < 12 A, class c(j) (C and S -> 0, N and P
// -> 1, O -> 2, H -> 3), shell s = 0..15 centred at mu_s = 1.5 + 0.7 s A
// with width sigma = 0.7 A:
//   D_i[16 c + s] = sum_j rho_j fc(r) exp(-(r - mu_s)^2 / (2 sigma^2)),
//   fc(r) = (cos(pi r / 12) + 1) / 2,
// rho_j the partner's intrinsic GB radius.  The network input is 80 wide:
// x[0..64) = log(1 + D), then 16 features of the atom itself: its class one-
// hot (4), rho~_i, its HCT scale s_i, rho~_i / R_cfa, log R_cfa, 0,
// log(rho~_i / R_cfa) and six zeros.  The output is
//   y = w4 . h3 + b4 + v . x[64..80)
// -- the 3 x 128 SiLU network plus a linear FP32 path on the self features,
// which keeps them at FP32 precision past the BF16 tensor-core products.
// The Coulomb-field baseline is the pairwise
// (Hawkins-Cramer-Truhlar) form of the Coulomb-field approximation over the
// same neighbours,
//   1/R_cfa = max(1/rho~_i - sum_j fc(r) I_HCT(r, rho~_i, s_j rho~_j), 1/30 A),
// and the learned radius is R = R_cfa exp(y), y the network output clamped
// to [-5, 5].
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "step_kernels.cuh"

namespace ogk {

constexpr int kLgbDesc = 64, kLgbIn = 80, kLgbHidden = 128;
constexpr double kLgbCutoff = 12.0;
// Parameters, FP32, in this order: W1[128x80] b1[128] W2[128x128] b2[128]
// W3[128x128] b3[128] w4[128] b4[1] v[16] (W row-major, out x in).
constexpr int kLgbOffW1 = 0;
constexpr int kLgbOffB1 = kLgbOffW1 + kLgbHidden * kLgbIn;
constexpr int kLgbOffW2 = kLgbOffB1 + kLgbHidden;
constexpr int kLgbOffB2 = kLgbOffW2 + kLgbHidden * kLgbHidden;
constexpr int kLgbOffW3 = kLgbOffB2 + kLgbHidden;
constexpr int kLgbOffB3 = kLgbOffW3 + kLgbHidden * kLgbHidden;
constexpr int kLgbOffW4 = kLgbOffB3 + kLgbHidden;
constexpr int kLgbOffB4 = kLgbOffW4 + kLgbHidden;
constexpr int kLgbOffV = kLgbOffB4 + 1;
constexpr int kLgbNSelf = kLgbIn - kLgbDesc;
constexpr int kLgbNParams = kLgbOffV + kLgbNSelf;

struct LgbDescArgs {
  const double* x;
  const double* y;
  const double* z;
  const int32_t* atom_sys;     // -1 for padding
  const int32_t* klass;        // descriptor class 0..3 per padded atom
  const double* rho;           // intrinsic radius
  const double* rho_tilde;     // rho - offset
  const double* srho;          // HCT scale * rho~
  const int2* sys_tiles;       // per system: (first tile, tile count)
  const double4* origin;       // per tile: centroid, w = bounding radius
  int32_t n_padded;
  float* xin;                  // n_padded x 80 network inputs (padding rows 0)
  double* r_cfa;               // n_padded (padding: 1)
};

// Descriptors and Coulomb-field radii of every atom (one 4-warp block per tile).
void launch_lgb_descriptors(const LgbDescArgs& a, cudaStream_t s);

// y = w4 . h3 + b4 + v . xself per row, R = r_cfa exp(clamp(y)) -> born_r
// (FP64) and the force pass's tile-SoA gb columns; padding atoms keep R = rho~.
void launch_lgb_radii(const AtomArrays& at, const float* h3, const float* xin, const float* params,
                      const double* r_cfa, cudaStream_t s);

// The whole network and the radii in one persistent tensor-core kernel
// (lgb_mlp.cu): same result as the three GEMM layers + launch_lgb_radii.
void launch_lgb_mlp_radii(const AtomArrays& at, const float* xin, const float* params, const double* r_cfa,
                          int32_t* error_flag, int n_sm, cudaStream_t s);
cudaError_t lgb_mlp_prepare();

// Judge: per system s (atoms [begin[s], end[s])), part[2s] = sum |Fa - Fb|^2
// and part[2s+1] = sum |Fb|^2 over two fixed-point force sets (kForceScale),
// one block per system in a fixed order.
void launch_lgb_force_error(const unsigned long long* fax, const unsigned long long* fay,
                            const unsigned long long* faz, const unsigned long long* fbx,
                            const unsigned long long* fby, const unsigned long long* fbz, const int32_t* begin,
                            const int32_t* end, int n_sys, double* part, cudaStream_t s);

// ---- training (row-major FP32 buffers, B rows)
// xb[B x 80], tb[B] = gathered rows idx[0..B) of x[n x 80], t[n]
void launch_lgb_gather(const float* x, const float* t, const int64_t* idx, int b, float* xb, float* tb,
                       cudaStream_t s);
// y = h3 w4 + b4 + xself v, loss partials, dy = 2 (y - t) / B, and
// dz3 = dy w4^T * silu'(z3); per-block loss partials in loss_part
void launch_lgb_head(const float* h3, const float* z3, const float* xb, const float* tb, const float* params, int b,
                     float* y, float* dy, float* dz3, float* loss_part, int loss_blocks, cudaStream_t s);
// g[k] = sum_r dy[r] xb[r, 64 + k]: the gradient of v
void launch_lgb_self_grad(const float* xb, const float* dy, int b, float* g_v, cudaStream_t s);
// g[k] = sum_r dy[r] h3[r, k] (k < 128) and g[128] = sum_r dy[r]: the w4, b4 gradient
void launch_lgb_head_grad(const float* h3, const float* dy, int b, float* g_w4b4, cudaStream_t s);
// column sums of dz [B x 128] -> g[128]
void launch_lgb_colsum(const float* dz, int b, float* g, cudaStream_t s);
// dz = dh * silu'(z), elementwise over n values
void launch_lgb_silu_bwd(const float* dh, const float* z, int64_t n, float* dz, cudaStream_t s);
// Adam (beta1 0.9, beta2 0.999, eps 1e-8) on all parameters, step t >= 1
void launch_lgb_adam(float* p, const float* g, float* m, float* v, int n, float lr, int t, cudaStream_t s);
// sum of loss partials -> out (one thread, fixed order)
void launch_lgb_sum(const float* part, int n, float* out, cudaStream_t s);

}  // namespace ogk
