// Per-atom / per-term kernels of one MD step.  See step_kernels.cuh.
#include <cmath>

#include "common.cuh"
#include "step_kernels.cuh"

namespace ogk {

namespace {

__device__ __forceinline__ double fixed_to_f(unsigned long long v) {
  return static_cast<double>(static_cast<long long>(v)) * kForceUnscale;
}

__device__ __forceinline__ bool atom_live(const AtomArrays& a, int i, int* sys) {
  if (i >= a.n_padded) return false;
  const int s = a.atom_sys[i];
  if (s < 0) return false;
  *sys = s;
  return (a.sys[s].status & kStatusDiverged) == 0;
}

// ------------------------------------------------------------------- pack
__device__ __forceinline__ void pack_atom(const AtomArrays& a, int i) {
  const int tile = i >> 5;
  // The tile's origin is the centroid of its real atoms and origin.w the
  // radius of its bounding sphere about it: the reference frame of the FP32
  // coordinates and the sphere every tile-level cull tests (cutoff lists,
  // descriptor partners, the SASA neighbour search).  The whole warp is one
  // tile: n_padded is a multiple of 32 and launches use whole warps.
  const bool real = a.atom_sys[i] >= 0;
  double sx = real ? a.x[i] : 0.0, sy = real ? a.y[i] : 0.0, sz = real ? a.z[i] : 0.0;
  for (int o = 16; o > 0; o >>= 1) {
    sx += __shfl_xor_sync(0xffffffffu, sx, o);
    sy += __shfl_xor_sync(0xffffffffu, sy, o);
    sz += __shfl_xor_sync(0xffffffffu, sz, o);
  }
  const int n_real = __popc(__ballot_sync(0xffffffffu, real));
  const double inv_n = n_real > 0 ? 1.0 / n_real : 0.0;
  const double ox = sx * inv_n, oy = sy * inv_n, oz = sz * inv_n;
  double rad = 0.0;
  if (a.atom_sys[i] >= 0) {
    const double dx = a.x[i] - ox, dy = a.y[i] - oy, dz = a.z[i] - oz;
    rad = sqrt(dx * dx + dy * dy + dz * dz);
  }
  for (int o = 16; o > 0; o >>= 1) rad = fmax(rad, __shfl_xor_sync(0xffffffffu, rad, o));
  if ((i & 31) == 0) a.origin[tile] = make_double4(ox, oy, oz, rad);
  if (a.atom_sys[i] >= 0) {
    a.pq[soa_index(i, 0)] = static_cast<float>(a.x[i] - ox);
    a.pq[soa_index(i, 1)] = static_cast<float>(a.y[i] - oy);
    a.pq[soa_index(i, 2)] = static_cast<float>(a.z[i] - oz);
    a.pq[soa_index(i, 3)] = static_cast<float>(a.q[i]);
  } else {
    // Padding: far from everything, no charge, no LJ (params are zero).
    a.pq[soa_index(i, 0)] = 1.0e6f + 16.0f * static_cast<float>(i & 31);
    a.pq[soa_index(i, 1)] = 1.0e6f;
    a.pq[soa_index(i, 2)] = 1.0e6f;
    a.pq[soa_index(i, 3)] = 0.0f;
  }
}

__device__ __forceinline__ void store_gb(const AtomArrays& a, int i, float r, float inv_r, float rt, float srho) {
  a.gb[soa_index(i, 0)] = r;
  a.gb[soa_index(i, 1)] = inv_r;
  a.gb[soa_index(i, 2)] = rt;
  a.gb[soa_index(i, 3)] = srho;
}

__global__ void k_pack(AtomArrays a, bool zero_acc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n_padded) return;
  pack_atom(a, i);
  if (zero_acc) {
    a.fx[i] = 0ull;
    a.fy[i] = 0ull;
    a.fz[i] = 0ull;
    a.born_sum[i] = 0ull;
  }
}

// ------------------------------------------------------------ Born radii
__global__ void k_born_finalize(AtomArrays a, const double* integral64, double* out_r, bool write_gb,
                                int32_t* clamp_count) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n_padded) return;
  const int sys = a.atom_sys[i];
  if (sys < 0) {
    if (write_gb) store_gb(a, i, 1.0f, 1.0f, 1.0f, 0.0f);
    out_r[i] = 1.0;
    return;
  }
  const double integral = integral64 ? integral64[i]
                                     : static_cast<double>(static_cast<long long>(a.born_sum[i])) * kBornUnscale;
  const double rt = a.rho_tilde[i];
  const double rho = a.rho[i];
  const double psi = integral * rt;
  const double arg = kObcAlpha * psi - kObcBeta * psi * psi + kObcGamma * psi * psi * psi;
  const double inv = 1.0 / rt - tanh(arg) / rho;
  const double floor_r = rt > 0.5 ? rt : 0.5;
  double r;
  if (inv <= 0.0 || !isfinite(inv)) {
    r = floor_r;
    if (clamp_count) atomicAdd(clamp_count + sys, 1);
  } else {
    r = 1.0 / inv;
    r = r > floor_r ? r : floor_r;
  }
  out_r[i] = r;
  if (write_gb)
    store_gb(a, i, static_cast<float>(r), static_cast<float>(1.0 / r), static_cast<float>(rt),
                  static_cast<float>(a.srho[i]));
}

// ----------------------------------------------------------------- bonded
struct D3 {
  double x, y, z;
};
__device__ __forceinline__ D3 operator-(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ D3 operator+(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ D3 operator*(D3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ D3 operator/(D3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ D3 neg(D3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ D3 cross(D3 a, D3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ double norm(D3 a) { return sqrt(dot(a, a)); }
__device__ __forceinline__ D3 ld(const BondedArgs& a, int i) { return {a.x[i], a.y[i], a.z[i]}; }
__device__ __forceinline__ void scatter(const BondedArgs& a, int i, D3 f) {
  if (!(isfinite(f.x) && isfinite(f.y) && isfinite(f.z))) atomicOr(a.sys_nonfinite + a.atom_sys[i], 1);
  add_fixed(a.fx + i, f.x, kForceScale);
  add_fixed(a.fy + i, f.y, kForceScale);
  add_fixed(a.fz + i, f.z, kForceScale);
}
__device__ __forceinline__ double wrap_pi(double d) {
  while (d > M_PI) d -= 2.0 * M_PI;
  while (d < -M_PI) d += 2.0 * M_PI;
  return d;
}

// energy/src/forces_bonded.rs:124-167
__device__ bool dihedral_gradient(D3 pa, D3 pb, D3 pc, D3 pd, D3* da, D3* db, D3* dc, D3* dd, double* phi) {
  const D3 b1 = pb - pa, b2 = pc - pb, b3 = pd - pc;
  const double b2n = norm(b2);
  if (b2n < 1e-9) return false;
  const D3 s = cross(b1, b2), t = cross(b2, b3);
  const double s2 = dot(s, s), t2 = dot(t, t);
  if (s2 < 1e-18 || t2 < 1e-18) return false;
  *da = s * (b2n / s2);
  *dd = neg(t) * (b2n / t2);
  const double inv = 1.0 / (b2n * b2n);
  const double f1 = dot(b1, b2) * inv, f2 = dot(b3, b2) * inv;
  *db = (*da) * (-(f1 + 1.0)) + (*dd) * f2;
  *dc = neg((*da + *db) + *dd);
  const D3 m1 = cross(s, b2 / b2n);
  *phi = atan2(dot(m1, t), dot(s, t));
  return true;
}

// geom/src/measure.rs:9-28
__device__ double measure_angle(D3 a, D3 b, D3 c) {
  D3 ba = a - b, bc = c - b;
  ba = ba / norm(ba);
  bc = bc / norm(bc);
  return acos(fmin(fmax(dot(ba, bc), -1.0), 1.0));
}
__device__ double measure_dihedral(D3 a, D3 b, D3 c, D3 d) {
  const D3 b0 = a - b;
  D3 b1 = c - b;
  b1 = b1 / norm(b1);
  const D3 b2 = d - c;
  const D3 v = b0 - b1 * dot(b0, b1);
  const D3 w = b2 - b1 * dot(b2, b1);
  return atan2(dot(cross(b1, v), w), dot(v, w));
}

template <bool kEnergy>
__global__ void k_bonded(BondedArgs a) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int n_all = a.n_bonds + a.n_angles + a.n_dihedrals + a.n_impropers;
  if (k >= n_all) return;
  const int slot = k;
  if (k < a.n_bonds) {  // forces_bonded.rs:47-71, bonded.rs:60-88
    const int2 ab = a.bond_atoms[k];
    const D3 d = ld(a, ab.y) - ld(a, ab.x);
    const double r = norm(d);
    const double dr = r - a.bond_r0[k];
    if (kEnergy) {
      a.energy[slot] = a.bond_k[k] * dr * dr * kKcalToKj;
    } else if (r >= 1e-9) {
      const double mag = (2.0 * a.bond_k[k] * dr) * kKcalToKj;
      const D3 f = d * (mag / r);
      scatter(a, ab.x, f);
      scatter(a, ab.y, neg(f));
    }
    return;
  }
  k -= a.n_bonds;
  if (k < a.n_angles) {  // forces_bonded.rs:79-118, bonded.rs:91-117
    const int4 q = a.angle_atoms[k];
    if (kEnergy) {
      const double d = measure_angle(ld(a, q.x), ld(a, q.y), ld(a, q.z)) - a.angle_t0[k];
      a.energy[slot] = a.angle_k[k] * d * d * kKcalToKj;
      return;
    }
    const D3 u = ld(a, q.x) - ld(a, q.y), v = ld(a, q.z) - ld(a, q.y);
    const double un = norm(u), vn = norm(v);
    if (un < 1e-9 || vn < 1e-9) return;
    const D3 uh = u / un, vh = v / vn;
    const double ct = fmin(fmax(dot(uh, vh), -1.0), 1.0);
    const double st = sqrt(1.0 - ct * ct);
    if (st < 1e-9) return;
    const double dv = 2.0 * a.angle_k[k] * (acos(ct) - a.angle_t0[k]);
    const double coeff = dv * kKcalToKj / st;
    const D3 fa = (vh - uh * ct) * (coeff / un);
    const D3 fc = (uh - vh * ct) * (coeff / vn);
    scatter(a, q.x, fa);
    scatter(a, q.y, neg(fa + fc));
    scatter(a, q.z, fc);
    return;
  }
  k -= a.n_angles;
  if (k < a.n_dihedrals) {  // forces_bonded.rs:174-205, bonded.rs:120-150
    const int4 q = a.dih_atoms[k];
    const int2 tr = a.dih_terms[k];
    if (kEnergy) {
      const double chi = measure_dihedral(ld(a, q.x), ld(a, q.y), ld(a, q.z), ld(a, q.w));
      double e = 0.0;
      for (int m = tr.x; m < tr.y; ++m) e += a.term_k[m] * (1.0 + cos(a.term_n[m] * chi - a.term_delta[m]));
      a.energy[slot] = e * kKcalToKj;
      return;
    }
    D3 da, db, dc, dd;
    double phi;
    if (!dihedral_gradient(ld(a, q.x), ld(a, q.y), ld(a, q.z), ld(a, q.w), &da, &db, &dc, &dd, &phi)) return;
    double dvdphi = 0.0;
    for (int m = tr.x; m < tr.y; ++m)
      dvdphi += -a.term_k[m] * static_cast<double>(a.term_n[m]) * sin(a.term_n[m] * phi - a.term_delta[m]);
    dvdphi *= kKcalToKj;
    scatter(a, q.x, neg(da * dvdphi));
    scatter(a, q.y, neg(db * dvdphi));
    scatter(a, q.z, neg(dc * dvdphi));
    scatter(a, q.w, neg(dd * dvdphi));
    return;
  }
  k -= a.n_dihedrals;
  {  // impropers: forces_bonded.rs:211-236, bonded.rs:153-191
    const int4 q = a.imp_atoms[k];
    if (kEnergy) {
      const double d =
          wrap_pi(measure_dihedral(ld(a, q.x), ld(a, q.y), ld(a, q.z), ld(a, q.w)) - a.imp_psi0[k]);
      a.energy[slot] = a.imp_k[k] * d * d * kKcalToKj;
      return;
    }
    D3 da, db, dc, dd;
    double om;
    if (!dihedral_gradient(ld(a, q.x), ld(a, q.y), ld(a, q.z), ld(a, q.w), &da, &db, &dc, &dd, &om)) return;
    const double dv = (2.0 * a.imp_k[k] * wrap_pi(om - a.imp_psi0[k])) * kKcalToKj;
    scatter(a, q.x, neg(da * dv));
    scatter(a, q.y, neg(db * dv));
    scatter(a, q.z, neg(dc * dv));
    scatter(a, q.w, neg(dd * dv));
  }
}

// ------------------------------------------------------------------ BAOAB
__global__ void k_step_pre(StepArgs p) {
  const AtomArrays& a = p.at;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  int sys;
  if (!atom_live(a, i, &sys)) return;
  const double c = (kAccel / a.mass[i]) * p.half_dt;
  double vx = a.vx[i] + fixed_to_f(a.fx[i]) * c;
  double vy = a.vy[i] + fixed_to_f(a.fy[i]) * c;
  double vz = a.vz[i] + fixed_to_f(a.fz[i]) * c;
  a.vx[i] = vx; a.vy[i] = vy; a.vz[i] = vz;
  const double x = a.x[i], y = a.y[i], z = a.z[i];
  if (p.use_shake) { a.rx[i] = x; a.ry[i] = y; a.rz[i] = z; }
  a.x[i] = x + vx * p.half_dt;
  a.y[i] = y + vy * p.half_dt;
  a.z[i] = z + vz * p.half_dt;
}

__device__ __forceinline__ void count_shake(const AtomArrays& a, int i, int sys) {
  if (a.local_idx[i] == 0) {
    SysState& s = a.sys[sys];
    if (s.shake_flag) {
      s.shake_failures += 1;
      s.status |= kStatusShakeFail;
      s.shake_flag = 0;
    }
  }
}

__global__ void k_step_mid(StepArgs p) {
  const AtomArrays& a = p.at;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  int sys;
  if (!atom_live(a, i, &sys)) return;
  double vx, vy, vz;
  if (p.use_shake) {
    vx = (a.x[i] - a.rx[i]) / p.half_dt;
    vy = (a.y[i] - a.ry[i]) / p.half_dt;
    vz = (a.z[i] - a.rz[i]) / p.half_dt;
    count_shake(a, i, sys);
  } else {
    vx = a.vx[i]; vy = a.vy[i]; vz = a.vz[i];
  }
  const SysState& s = a.sys[sys];
  // O step (langevin.rs:260-271) with Philox noise keyed by (system, step, atom).
  const unsigned long long step = static_cast<unsigned long long>(s.steps) + 1ull;
  const U4 r = philox4x32_10(U4{static_cast<uint32_t>(a.local_idx[i]), static_cast<uint32_t>(step),
                                 static_cast<uint32_t>(step >> 32), static_cast<uint32_t>(sys)},
                              p.seed_lo, p.seed_hi);
  const double m1 = sqrt(-2.0 * log(u32_to_open01(r.x)));
  const double m2 = sqrt(-2.0 * log(u32_to_open01(r.z)));
  double s1, c1, s2, c2;
  sincospi(2.0 * (static_cast<double>(r.y) * (1.0 / 4294967296.0)), &s1, &c1);
  sincospi(2.0 * (static_cast<double>(r.w) * (1.0 / 4294967296.0)), &s2, &c2);
  const double one_minus_a2 = 1.0 - p.alpha * p.alpha;
  const double sigma = sqrt(one_minus_a2 * s.kbt * s.dof_corr * kAccel / a.mass[i]);
  vx = p.alpha * vx + sigma * (m1 * c1);
  vy = p.alpha * vy + sigma * (m1 * s1);
  vz = p.alpha * vz + sigma * (m2 * c2);
  a.vx[i] = vx; a.vy[i] = vy; a.vz[i] = vz;
  const double x = a.x[i], y = a.y[i], z = a.z[i];
  if (p.use_shake) { a.rx[i] = x; a.ry[i] = y; a.rz[i] = z; }
  a.x[i] = x + vx * p.half_dt;
  a.y[i] = y + vy * p.half_dt;
  a.z[i] = z + vz * p.half_dt;
}

__global__ void k_step_post(StepArgs p) {
  const AtomArrays& a = p.at;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n_padded) return;
  int sys;
  if (p.use_shake && atom_live(a, i, &sys)) {
    a.vx[i] = (a.x[i] - a.rx[i]) / p.half_dt;
    a.vy[i] = (a.y[i] - a.ry[i]) / p.half_dt;
    a.vz[i] = (a.z[i] - a.rz[i]) / p.half_dt;
    count_shake(a, i, sys);
  }
  pack_atom(a, i);
  a.fx[i] = 0ull;
  a.fy[i] = 0ull;
  a.fz[i] = 0ull;
  a.born_sum[i] = 0ull;
}

__global__ void k_step_end(StepArgs p) {
  const AtomArrays& a = p.at;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  int sys;
  if (!atom_live(a, i, &sys)) return;
  const double c = (kAccel / a.mass[i]) * p.half_dt;
  const double vx = a.vx[i] + fixed_to_f(a.fx[i]) * c;
  const double vy = a.vy[i] + fixed_to_f(a.fy[i]) * c;
  const double vz = a.vz[i] + fixed_to_f(a.fz[i]) * c;
  a.vx[i] = vx; a.vy[i] = vy; a.vz[i] = vz;
  if (!(isfinite(vx) && isfinite(vy) && isfinite(vz)) || a.sys_nonfinite[sys])
    atomicOr(&a.sys[sys].status, kStatusDiverged);
  if (a.local_idx[i] == 0) a.sys[sys].steps += 1;
}

// ------------------------------------------------------------------ SHAKE
// One thread per heavy-atom cluster (an X-H constraint group); Gauss-Seidel
// passes in the reference's constraint order until every constraint of the
// cluster is inside tolerance (shake.rs:86-125).  Clusters share no atom, so
// this equals the reference's global passes.
__global__ void k_shake(ShakeArgs a) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.n_clusters) return;
  const int sys = a.cluster_sys[c];
  if (a.sys[sys].status & kStatusDiverged) return;
  const int b = a.cluster_start[c], e = a.cluster_start[c + 1];
  bool converged = false;
  for (int iter = 0; iter < a.max_iters && !converged; ++iter) {
    double max_err = 0.0;
    for (int k = b; k < e; ++k) {
      const int i = a.cons_atoms[k].x, j = a.cons_atoms[k].y;
      const double rnx = a.x[i] - a.x[j], rny = a.y[i] - a.y[j], rnz = a.z[i] - a.z[j];
      const double err = (rnx * rnx + rny * rny + rnz * rnz) - a.cons_d2[k];
      if (fabs(err) > max_err) max_err = fabs(err);
      if (fabs(err) < a.tol_sq) continue;
      const double rox = a.rx[i] - a.rx[j], roy = a.ry[i] - a.ry[j], roz = a.rz[i] - a.rz[j];
      const double dotv = rnx * rox + rny * roy + rnz * roz;
      const double denom = 2.0 * (a.inv_mass[i] + a.inv_mass[j]) * dotv;
      if (fabs(denom) < 1e-18) continue;
      const double lambda = err / denom;
      const double dx = rox * lambda, dy = roy * lambda, dz = roz * lambda;
      a.x[i] -= dx * a.inv_mass[i]; a.y[i] -= dy * a.inv_mass[i]; a.z[i] -= dz * a.inv_mass[i];
      a.x[j] += dx * a.inv_mass[j]; a.y[j] += dy * a.inv_mass[j]; a.z[j] += dz * a.inv_mass[j];
    }
    converged = max_err < a.tol_sq;
  }
  if (!converged) atomicOr(&a.sys[sys].shake_flag, 1);
}

// ------------------------------------------------------------- reductions
constexpr int kRedThreads = 256;

__device__ double block_sum_fixed_order(double v) {
  __shared__ double sh[kRedThreads];
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int w = kRedThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  return sh[0];
}

__global__ void k_segment_sum(const double* v, const int32_t* begin, const int32_t* end, double* out) {
  const int s = blockIdx.x;
  double acc = 0.0;
  for (int k = begin[s] + threadIdx.x; k < end[s]; k += kRedThreads) acc += v[k];
  const double tot = block_sum_fixed_order(acc);
  if (threadIdx.x == 0) out[s] = tot;
}

__global__ void k_kinetic(AtomArrays a, const int32_t* begin, const int32_t* end, double* out) {
  const int s = blockIdx.x;
  double acc = 0.0;
  for (int k = begin[s] + threadIdx.x; k < end[s]; k += kRedThreads)
    acc += a.mass[k] * (a.vx[k] * a.vx[k] + a.vy[k] * a.vy[k] + a.vz[k] * a.vz[k]);
  const double tot = block_sum_fixed_order(acc);
  if (threadIdx.x == 0) out[s] = 0.5 * tot / kAccel;
}

// ------------------------------------------------------ replica exchange
// Per system the potential energy og_compute_energies reports (bonded +
// LJ/RF + GB, kJ/mol), from the per-atom and per-term FP64 energies: each
// term summed exactly as k_segment_sum does, then combined in the same
// order as the host, so the total is bit-identical to og_compute_energies'.
__global__ void k_remd_totals(const double* e_lj, const double* e_coul, const double* e_gb, const double* e_self,
                              const double* bonded_e, const int32_t* begin, const int32_t* end, int n_sys,
                              double* total) {
  const int s = blockIdx.x;
  double part[8];
  const double* per_atom[4] = {e_lj, e_coul, e_gb, e_self};
  for (int t = 0; t < 8; ++t) {
    const int seg = t < 4 ? s : (t - 3) * n_sys + s;
    const double* v = t < 4 ? per_atom[t] : bonded_e;
    double acc = 0.0;
    for (int k = begin[seg] + threadIdx.x; k < end[seg]; k += kRedThreads) acc += v[k];
    part[t] = block_sum_fixed_order(acc);
    __syncthreads();  // the next sum reuses the shared buffer
  }
  if (threadIdx.x == 0) {
    const double lj = 0.5 * part[0] * kKcalToKj, coul = 0.5 * part[1] * kKcalToKj;
    const double gb_pair = 0.5 * part[2] * kKcalToKj, gb_self = part[3] * kKcalToKj;
    const double gb = gb_self + gb_pair;
    total[s] = part[4] + part[5] + part[6] + part[7] + lj + coul + gb;
  }
}

// One swap round: neighbouring temperature slots (pi, pi + 1), pi = parity,
// parity + 2, ... (remd.rs:425-474).  Slot pi holds system sys_of_slot[pi]
// at temperature temps[pi]; an accepted exchange swaps the two systems'
// slots (their temperatures) and marks their velocities for rescaling by
// sqrt(T_new / T_old).  The uniform of pair pi in round r is Philox keyed by
// (seed, r, pi).  One thread: the pairs are few and the decisions ordered.
__global__ void k_remd_swap(SysState* sys, int32_t* sys_of_slot, const double* temps, const double* total,
                            int n_slots, int parity, uint64_t seed, uint32_t round, long long* attempts,
                            long long* accepts, double* vscale) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int k = 0; k < n_slots; ++k) vscale[k] = 1.0;
  for (int pi = parity; pi + 1 < n_slots; pi += 2) {
    const int a = sys_of_slot[pi], b = sys_of_slot[pi + 1];
    if ((sys[a].status | sys[b].status) & kStatusDiverged) continue;
    attempts[pi] += 1;
    const U4 r = philox4x32_10(U4{static_cast<uint32_t>(pi), round, 0x52454D44u, 0u}, static_cast<uint32_t>(seed),
                               static_cast<uint32_t>(seed >> 32));
    const double u = u32_to_open01(r.x);
    const double ta = temps[pi], tb = temps[pi + 1];
    const double delta = (1.0 / (kBoltzmann * ta) - 1.0 / (kBoltzmann * tb)) * (total[a] - total[b]);
    const double p_acc = delta >= 0.0 ? 1.0 : exp(delta);
    if (u < p_acc) {
      accepts[pi] += 1;
      sys_of_slot[pi] = b;
      sys_of_slot[pi + 1] = a;
      sys[a].temperature = tb;
      sys[a].kbt = kBoltzmann * tb;
      sys[b].temperature = ta;
      sys[b].kbt = kBoltzmann * ta;
      vscale[a] = sqrt(tb / ta);
      vscale[b] = sqrt(ta / tb);
    }
  }
}

__global__ void k_remd_rescale(AtomArrays a, const double* vscale) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n_padded) return;
  const int s = a.atom_sys[i];
  if (s < 0) return;
  const double f = vscale[s];
  if (f == 1.0) return;
  a.vx[i] *= f;
  a.vy[i] *= f;
  a.vz[i] *= f;
}

inline int blocks_for(int n, int bs) { return (n + bs - 1) / bs; }

}  // namespace

void launch_pack(const AtomArrays& a, bool zero_acc, cudaStream_t s) {
  k_pack<<<blocks_for(a.n_padded, 256), 256, 0, s>>>(a, zero_acc);
}

void launch_born_finalize(const AtomArrays& a, const double* integral64, double* out_r, bool write_gb,
                          int32_t* clamp_count, cudaStream_t s) {
  k_born_finalize<<<blocks_for(a.n_padded, 256), 256, 0, s>>>(a, integral64, out_r, write_gb, clamp_count);
}

__global__ void k_swap_systems(AtomArrays a, int32_t ba, int32_t bb, int32_t n, double scale_a, double scale_b) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int i = ba + k, j = bb + k;
  double t;
  t = a.x[i]; a.x[i] = a.x[j]; a.x[j] = t;
  t = a.y[i]; a.y[i] = a.y[j]; a.y[j] = t;
  t = a.z[i]; a.z[i] = a.z[j]; a.z[j] = t;
  const double vxi = a.vx[i], vyi = a.vy[i], vzi = a.vz[i];
  a.vx[i] = a.vx[j] * scale_a; a.vy[i] = a.vy[j] * scale_a; a.vz[i] = a.vz[j] * scale_a;
  a.vx[j] = vxi * scale_b; a.vy[j] = vyi * scale_b; a.vz[j] = vzi * scale_b;
  unsigned long long u;
  u = a.fx[i]; a.fx[i] = a.fx[j]; a.fx[j] = u;
  u = a.fy[i]; a.fy[i] = a.fy[j]; a.fy[j] = u;
  u = a.fz[i]; a.fz[i] = a.fz[j]; a.fz[j] = u;
  double r = a.born_r[i]; a.born_r[i] = a.born_r[j]; a.born_r[j] = r;
}

void launch_swap_systems(const AtomArrays& a, int32_t begin_a, int32_t begin_b, int32_t n, double scale_a,
                         double scale_b, cudaStream_t s) {
  if (n > 0) k_swap_systems<<<blocks_for(n, 256), 256, 0, s>>>(a, begin_a, begin_b, n, scale_a, scale_b);
}

void launch_bonded_forces(const BondedArgs& a, cudaStream_t s) {
  const int n = a.n_bonds + a.n_angles + a.n_dihedrals + a.n_impropers;
  if (n > 0) k_bonded<false><<<blocks_for(n, 128), 128, 0, s>>>(a);
}

void launch_bonded_energies(const BondedArgs& a, cudaStream_t s) {
  const int n = a.n_bonds + a.n_angles + a.n_dihedrals + a.n_impropers;
  if (n > 0) k_bonded<true><<<blocks_for(n, 128), 128, 0, s>>>(a);
}

void launch_step_pre(const StepArgs& a, cudaStream_t s) {
  k_step_pre<<<blocks_for(a.at.n_padded, 256), 256, 0, s>>>(a);
}
void launch_step_mid(const StepArgs& a, cudaStream_t s) {
  k_step_mid<<<blocks_for(a.at.n_padded, 256), 256, 0, s>>>(a);
}
void launch_step_post(const StepArgs& a, cudaStream_t s) {
  k_step_post<<<blocks_for(a.at.n_padded, 256), 256, 0, s>>>(a);
}
void launch_step_end(const StepArgs& a, cudaStream_t s) {
  k_step_end<<<blocks_for(a.at.n_padded, 256), 256, 0, s>>>(a);
}

void launch_shake(const ShakeArgs& a, cudaStream_t s) {
  if (a.n_clusters > 0) k_shake<<<blocks_for(a.n_clusters, 128), 128, 0, s>>>(a);
}

void launch_segment_sum(const double* v, const int32_t* begin, const int32_t* end, int32_t n_seg, double* out,
                        cudaStream_t s) {
  if (n_seg > 0) k_segment_sum<<<n_seg, kRedThreads, 0, s>>>(v, begin, end, out);
}

void launch_kinetic(const AtomArrays& a, const int32_t* begin, const int32_t* end, int32_t n_sys, double* out,
                    cudaStream_t s) {
  if (n_sys > 0) k_kinetic<<<n_sys, kRedThreads, 0, s>>>(a, begin, end, out);
}

void launch_remd_round(const AtomArrays& a, const RemdArgs& r, int parity, uint32_t round, cudaStream_t s) {
  if (r.n_slots < 2) return;
  k_remd_totals<<<r.n_slots, kRedThreads, 0, s>>>(r.e_lj, r.e_coul, r.e_gb, r.e_self, r.bonded_e, r.seg_begin,
                                                  r.seg_end, r.n_slots, r.total);
  k_remd_swap<<<1, 32, 0, s>>>(r.sys, r.sys_of_slot, r.temps, r.total, r.n_slots, parity, r.seed, round, r.attempts,
                               r.accepts, r.vscale);
  k_remd_rescale<<<blocks_for(a.n_padded, 256), 256, 0, s>>>(a, r.vscale);
}

namespace {

// One thread per atom; it owns its accumulators here (the force kernels
// have finished in stream order), so a plain add suffices.
__global__ void k_tunnel(AtomArrays a, TunnelParams t) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n_padded || a.atom_sys[i] < 0) return;
  const double rx = a.x[i] - t.ox, ry = a.y[i] - t.oy, rz = a.z[i] - t.oz;
  const double along = rx * t.dx + ry * t.dy + rz * t.dz;
  if (along < 0.0 || along > t.length) return;
  const double px = rx - t.dx * along, py = ry - t.dy * along, pz = rz - t.dz * along;
  const double d = sqrt(px * px + py * py + pz * pz);
  if (!(d > t.radius)) return;
  const double s = -t.k * (d - t.radius) / d;
  a.fx[i] += static_cast<unsigned long long>(__double2ll_rn(s * px * kForceScale));
  a.fy[i] += static_cast<unsigned long long>(__double2ll_rn(s * py * kForceScale));
  a.fz[i] += static_cast<unsigned long long>(__double2ll_rn(s * pz * kForceScale));
}

}  // namespace

void launch_tunnel(const AtomArrays& a, const TunnelParams& t, cudaStream_t s) {
  k_tunnel<<<blocks_for(a.n_padded, 256), 256, 0, s>>>(a, t);
}

}  // namespace ogk
