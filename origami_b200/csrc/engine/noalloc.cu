// og_gb_energy_noalloc: the GB solvation energy of one system computed
// without any device allocation.
//
// The FP64 energy path of the engine (pair_fp64.cu) needs scratch buffers
// (per-atom Born radii, per-atom partial sums) that the engine cudaMallocs at
// finalize time.  This entry point is for callers that cannot call cudaMalloc
// at the point where they need the energy -- for example a host whose device
// memory is entirely reserved up front by another framework's caching
// allocator, or a latency-critical loop that forbids allocation (and the
// device synchronisation cudaMalloc/cudaFree imply) after start-up.  Its
// scratch is a fixed array in the library's own device image instead:
//
//   g_noalloc_scratch: kNoAllocMaxAtoms Born radii + 2 partial sums per block
//                      (16 384 + 128 doubles, ~129 KiB on every GPU that
//                      loads the library, held until the process exits).
//
// The driver places that array (and the three kernels' code) in device
// memory when it loads this file's module, which with CUDA's default lazy
// loading happens at the first use, not at library load.  A call with
// n_atoms = 0 and every pointer NULL does only that set-up -- loads the
// module and resolves the array's address on the current device -- so a
// caller whose memory another allocator will reserve makes that call first.
//
// Host code cannot use the array's name as a device address, so each call
// looks the address up with cudaGetSymbolAddress with the target device
// current (the lookup allocates nothing once the module is loaded), which
// also keeps the address right after a cudaDeviceReset has replaced the
// context.  A call issued while its stream is being captured does not look
// anything up: it uses the address the last call outside capture on that
// device found.  Every call shares the one array: calls whose kernels
// overlap on the GPU (two streams, or two host threads) race and must be
// ordered by the caller.  Nothing in the scratch needs to start at zero --
// every element a call reads is written earlier in the same call.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../../include/origami_gpu.h"
#include "../host/status.h"
#include "common.cuh"

namespace {

constexpr int kNoAllocMaxAtoms = OG_NOALLOC_MAX_ATOMS;
constexpr int kThreads = 256;
constexpr int kMaxBlocks = (kNoAllocMaxAtoms + kThreads - 1) / kThreads;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocMaxAtoms + 2 * kMaxBlocks];

std::mutex g_mu;
double* g_scratch_ptr[kMaxDevices] = {nullptr};

// energy/src/gb.rs:347-369.
__device__ double descreen(double r, double rho_i, double s_rho_j) {
  if (r + s_rho_j <= rho_i) return 0.0;
  const double l = (r - s_rho_j < rho_i) ? rho_i : r - s_rho_j;
  const double u = r + s_rho_j;
  if (u <= 0.0 || l <= 0.0) return 0.0;
  const double inv_l = 1.0 / l, inv_u = 1.0 / u;
  const double term1 = 0.5 * (inv_l - inv_u);
  const double term2 = (r / 4.0) * (inv_u * inv_u - inv_l * inv_l);
  const double term3 = (1.0 / (2.0 * r)) * log(l / u);
  const double term4 = (s_rho_j * s_rho_j - r * r) / (4.0 * r) * (inv_u * inv_u - inv_l * inv_l);
  return term1 + term2 + term3 + term4;
}

// Effective Born radius of atom i (gb.rs:100-144, OBC-II map and clamp :326-341).
__global__ void k_noalloc_radii(const double* __restrict__ xyz, const double* __restrict__ rho,
                                const double* __restrict__ scale, int n, double born_c2, double* __restrict__ radii) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double xi = xyz[3 * i], yi = xyz[3 * i + 1], zi = xyz[3 * i + 2];
  const double rt = rho[i] - ogk::kObcOffset;
  double integral = 0.0;
  for (int j = 0; j < n; ++j) {
    if (j == i) continue;
    const double dx = xyz[3 * j] - xi, dy = xyz[3 * j + 1] - yi, dz = xyz[3 * j + 2] - zi;
    const double r2 = dx * dx + dy * dy + dz * dz;
    if (r2 > born_c2 || r2 < 1e-18) continue;
    integral += descreen(sqrt(r2), rt, scale[j] * (rho[j] - ogk::kObcOffset));
  }
  const double psi = integral * rt;
  const double arg = ogk::kObcAlpha * psi - ogk::kObcBeta * psi * psi + ogk::kObcGamma * psi * psi * psi;
  const double inv = 1.0 / rt - tanh(arg) / rho[i];
  const double floor_r = rt > 0.5 ? rt : 0.5;
  double r = floor_r;
  if (inv > 0.0 && isfinite(inv)) {
    r = 1.0 / inv;
    r = r > floor_r ? r : floor_r;
  }
  radii[i] = r;
}

// Self term of atom i and its pair terms with j > i (gb.rs:146-182), summed
// per block in a fixed order into partial[2 * block + {0, 1}] (kcal/mol).
__global__ void k_noalloc_energy(const double* __restrict__ xyz, const double* __restrict__ q,
                                 const double* __restrict__ radii, int n, double* __restrict__ partial) {
  __shared__ double s_self[kThreads], s_pair[kThreads];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const double pref = -0.5 * (1.0 - 1.0 / ogk::kEpsWater) * ogk::kCoulomb;
  double self_e = 0.0, pair_e = 0.0;
  if (i < n) {
    const double qi = q[i], Ri = radii[i];
    if (qi != 0.0) self_e = pref * (qi * qi) / Ri;
    const double xi = xyz[3 * i], yi = xyz[3 * i + 1], zi = xyz[3 * i + 2];
    for (int j = i + 1; j < n; ++j) {
      const double qq = qi * q[j];
      if (qq == 0.0) continue;
      const double dx = xyz[3 * j] - xi, dy = xyz[3 * j + 1] - yi, dz = xyz[3 * j + 2] - zi;
      const double r2 = dx * dx + dy * dy + dz * dz;
      const double rp = Ri * radii[j];
      pair_e += 2.0 * pref * qq / sqrt(r2 + rp * exp(-r2 / (4.0 * rp)));
    }
  }
  s_self[threadIdx.x] = self_e;
  s_pair[threadIdx.x] = pair_e;
  __syncthreads();
  for (int w = kThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      s_self[threadIdx.x] += s_self[threadIdx.x + w];
      s_pair[threadIdx.x] += s_pair[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    partial[2 * blockIdx.x] = s_self[0];
    partial[2 * blockIdx.x + 1] = s_pair[0];
  }
}

__global__ void k_noalloc_total(const double* __restrict__ partial, int n_blocks, double* __restrict__ out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double self_e = 0.0, pair_e = 0.0;
  for (int b = 0; b < n_blocks; ++b) {
    self_e += partial[2 * b];
    pair_e += partial[2 * b + 1];
  }
  out[0] = (self_e + pair_e) * ogk::kKcalToKj;
  out[1] = self_e * ogk::kKcalToKj;
  out[2] = pair_e * ogk::kKcalToKj;
}

// Loads this module on the current device (under lazy loading the driver
// places the scratch array and the kernels' code at this point) and returns
// the scratch array's device address there.  Outside stream capture the
// address is looked up afresh and cached per device; inside capture the
// cached address is used, since a lookup could have to load the module.
og_status scratch_address(cudaStream_t stream, double** out) {
  int dev = 0;
  cudaError_t err = cudaGetDevice(&dev);
  if (err != cudaSuccess) return og_fail(OG_E_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(err));
  if (dev < 0 || dev >= kMaxDevices) return og_fail(OG_E_UNSUPPORTED, "device index beyond the supported range");
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  err = cudaStreamIsCapturing(stream, &cap);
  if (err != cudaSuccess) return og_fail(OG_E_CUDA, std::string("cudaStreamIsCapturing: ") + cudaGetErrorString(err));
  std::lock_guard<std::mutex> lock(g_mu);
  if (cap != cudaStreamCaptureStatusNone) {
    if (!g_scratch_ptr[dev])
      return og_fail(OG_E_STATE, "og_gb_energy_noalloc: first call on this device made during stream capture; "
                                 "make a set-up call (n_atoms = 0, NULL pointers) before capturing");
    *out = g_scratch_ptr[dev];
    return OG_OK;
  }
  cudaFuncAttributes attr;
  const void* kernels[] = {reinterpret_cast<const void*>(&k_noalloc_radii),
                           reinterpret_cast<const void*>(&k_noalloc_energy),
                           reinterpret_cast<const void*>(&k_noalloc_total)};
  for (const void* k : kernels) {
    err = cudaFuncGetAttributes(&attr, k);
    if (err != cudaSuccess)
      return og_fail(OG_E_CUDA, std::string("cudaFuncGetAttributes: ") + cudaGetErrorString(err));
  }
  void* p = nullptr;
  err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (err != cudaSuccess || !p)
    return og_fail(OG_E_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(err));
  g_scratch_ptr[dev] = static_cast<double*>(p);
  *out = g_scratch_ptr[dev];
  return OG_OK;
}

}  // namespace

extern "C" og_status og_gb_energy_noalloc(const double* xyz, const double* charge, const double* gb_rho,
                                          const double* gb_scale, int32_t n_atoms, double born_cutoff,
                                          double* energy_out, void* stream) {
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double* scratch = nullptr;
  if (n_atoms == 0 && !xyz && !charge && !gb_rho && !gb_scale && !energy_out) return scratch_address(s, &scratch);
  if (!xyz || !charge || !gb_rho || !gb_scale || !energy_out) return og_fail(OG_E_BADARG, "null argument");
  if (n_atoms < 1 || n_atoms > kNoAllocMaxAtoms)
    return og_fail(OG_E_BADARG, "og_gb_energy_noalloc: n_atoms must be in [1, " +
                                    std::to_string(kNoAllocMaxAtoms) + "], got " + std::to_string(n_atoms));
  og_status st = scratch_address(s, &scratch);
  if (st != OG_OK) return st;
  double* radii = scratch;
  double* partial = scratch + kNoAllocMaxAtoms;
  const double c2 = (!(born_cutoff > 0.0) || born_cutoff >= 1e30) ? static_cast<double>(INFINITY)
                                                                   : born_cutoff * born_cutoff;
  const int blocks = (n_atoms + kThreads - 1) / kThreads;
  k_noalloc_radii<<<blocks, kThreads, 0, s>>>(xyz, gb_rho, gb_scale, n_atoms, c2, radii);
  k_noalloc_energy<<<blocks, kThreads, 0, s>>>(xyz, charge, radii, n_atoms, partial);
  k_noalloc_total<<<1, 32, 0, s>>>(partial, blocks, energy_out);
  const cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return og_fail(OG_E_CUDA, std::string("og_gb_energy_noalloc: ") + cudaGetErrorString(err));
  return OG_OK;
}
