// og_engine_*: the device half of the C ABI.
//
// An engine holds any number of systems (REMD replicas of one chain or
// independent chains of different lengths) concatenated in one padded atom
// space: every system starts on a 32-atom tile boundary, so a tile never
// straddles two systems.  Pair work is a list of (i-block, j-tile range)
// items; bonded terms, SHAKE clusters and per-system state are flat arrays
// with global atom indices.  One MD step is a fixed sequence of launches that
// is captured once into a CUDA graph and replayed.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <numeric>
#include <set>
#include <string>
#include <vector>

#include "../../../include/origami_gpu.h"
#include "../host/pdb.h"
#include "../host/status.h"
#include "common.cuh"
#include "lgb.cuh"
#include "pair_kernels.cuh"
#include "sasa.cuh"
#include "state.cuh"
#include "tc_gemm.cuh"
#include "step_kernels.cuh"

namespace ogk {
}

namespace {

using ogk::kTile;

bool no_cutoff(double c) { return !(c > 0.0) || c >= 1e30; }

og_status cuda_fail(cudaError_t e, const char* what) {
  return og_fail(OG_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define OG_CUDA(call)                                   \
  do {                                                  \
    cudaError_t _e = (call);                            \
    if (_e != cudaSuccess) return cuda_fail(_e, #call); \
  } while (0)

template <class T>
struct DVec {
  T* p = nullptr;
  size_t n = 0, cap = 0;
  ~DVec() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
    cap = 0;
  }
  cudaError_t alloc(size_t count) {
    release();
    n = count;
    cap = count;
    if (count == 0) return cudaSuccess;
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&p), count * sizeof(T));
    // OG_DEBUG_POISON=1 fills new buffers with 0xFF bytes (NaN as float or
    // double) so a read before the first write shows up as a non-finite result.
    // The fill runs on the legacy default stream, which does not order against
    // the engine's non-blocking stream, so it is waited for before the buffer
    // is handed out (else it could land after the buffer's first write).
    if (e == cudaSuccess && poison_enabled()) {
      e = cudaMemset(p, 0xFF, count * sizeof(T));
      if (e == cudaSuccess) e = cudaDeviceSynchronize();
    }
    return e;
  }
  static bool poison_enabled() {
    const char* v = std::getenv("OG_DEBUG_POISON");
    return v && v[0] == '1';
  }
  cudaError_t upload(const std::vector<T>& h, cudaStream_t s) {
    cudaError_t e = alloc(h.size());
    if (e != cudaSuccess || h.empty()) return e;
    return cudaMemcpyAsync(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, s);
  }
  // Resizes to `count` elements keeping the first min(n, count) on the
  // device; a larger buffer (half again as large, so that a run of small
  // appends reallocates rarely) is made only when the capacity is exceeded.
  cudaError_t grow(size_t count, cudaStream_t s) {
    if (count <= cap && p) {
      n = count;
      return cudaSuccess;
    }
    DVec<T> fresh;
    cudaError_t e = fresh.alloc(std::max(count, cap + cap / 2));
    if (e == cudaSuccess && n > 0)
      e = cudaMemcpyAsync(fresh.p, p, n * sizeof(T), cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // the old buffer is read until here
    if (e != cudaSuccess) return e;
    std::swap(p, fresh.p);
    std::swap(cap, fresh.cap);
    n = count;
    return cudaSuccess;  // `fresh` frees the old buffer
  }
  // h[from, h.size()) to the same positions on the device (grown to
  // h.size() elements first); h[0, from) is taken to be there already.
  cudaError_t upload_tail(const std::vector<T>& h, size_t from, cudaStream_t s) {
    cudaError_t e = grow(h.size(), s);
    if (e != cudaSuccess || from >= h.size()) return e;
    return cudaMemcpyAsync(p + from, h.data() + from, (h.size() - from) * sizeof(T), cudaMemcpyHostToDevice, s);
  }
  cudaError_t upload_range(const std::vector<T>& h, size_t from, size_t to, cudaStream_t s) {
    if (from >= to) return cudaSuccess;
    return cudaMemcpyAsync(p + from, h.data() + from, (to - from) * sizeof(T), cudaMemcpyHostToDevice, s);
  }
};

struct TopoCopy {
  int n = 0;
  std::vector<double> charge, rmin, eps, rmin14, eps14, rho, scale, mass;
  std::vector<int32_t> element;
  std::vector<int32_t> bonds, angles, dihedrals, dih_start, term_n, impropers, excl, cons;
  std::vector<double> bond_k, bond_r0, angle_k, angle_t0, term_k, term_delta, imp_k, imp_psi0, cons_d;
  std::vector<int8_t> excl_kind;
};

template <class T>
std::vector<T> copy_arr(const T* p, size_t n) {
  return (p && n) ? std::vector<T>(p, p + n) : std::vector<T>();
}

og_status copy_topology(const og_topology* t, TopoCopy* c) {
  const int n = t->n_atoms;
  if (n <= 0) return og_fail(OG_E_BADARG, "topology has no atoms");
  if (!t->charge || !t->rmin_half || !t->epsilon || !t->rmin_half_14 || !t->epsilon_14 || !t->gb_rho ||
      !t->gb_scale || !t->mass || !t->element)
    return og_fail(OG_E_BADARG, "topology per-atom array missing");
  c->n = n;
  c->charge = copy_arr(t->charge, n);
  c->rmin = copy_arr(t->rmin_half, n);
  c->eps = copy_arr(t->epsilon, n);
  c->rmin14 = copy_arr(t->rmin_half_14, n);
  c->eps14 = copy_arr(t->epsilon_14, n);
  c->rho = copy_arr(t->gb_rho, n);
  c->scale = copy_arr(t->gb_scale, n);
  c->mass = copy_arr(t->mass, n);
  c->element = copy_arr(t->element, n);
  c->bonds = copy_arr(t->bond_atoms, 2 * static_cast<size_t>(t->n_bonds));
  c->bond_k = copy_arr(t->bond_k, t->n_bonds);
  c->bond_r0 = copy_arr(t->bond_r0, t->n_bonds);
  c->angles = copy_arr(t->angle_atoms, 3 * static_cast<size_t>(t->n_angles));
  c->angle_k = copy_arr(t->angle_k, t->n_angles);
  c->angle_t0 = copy_arr(t->angle_theta0, t->n_angles);
  c->dihedrals = copy_arr(t->dihedral_atoms, 4 * static_cast<size_t>(t->n_dihedrals));
  c->dih_start = copy_arr(t->dihedral_term_start, static_cast<size_t>(t->n_dihedrals) + 1);
  c->term_k = copy_arr(t->term_k, t->n_dihedral_terms);
  c->term_n = copy_arr(t->term_n, t->n_dihedral_terms);
  c->term_delta = copy_arr(t->term_delta, t->n_dihedral_terms);
  c->impropers = copy_arr(t->improper_atoms, 4 * static_cast<size_t>(t->n_impropers));
  c->imp_k = copy_arr(t->improper_k, t->n_impropers);
  c->imp_psi0 = copy_arr(t->improper_psi0, t->n_impropers);
  c->excl = copy_arr(t->exclusion_atoms, 2 * static_cast<size_t>(t->n_exclusions));
  c->excl_kind = copy_arr(t->exclusion_kind, t->n_exclusions);
  c->cons = copy_arr(t->constraint_atoms, 2 * static_cast<size_t>(t->n_constraints));
  c->cons_d = copy_arr(t->constraint_length, t->n_constraints);
  if (t->n_dihedrals > 0 && c->dih_start.back() != t->n_dihedral_terms)
    return og_fail(OG_E_BADARG, "dihedral_term_start does not end at n_dihedral_terms");
  auto bad_idx = [n](const std::vector<int32_t>& v) {
    for (int32_t k : v)
      if (k < 0 || k >= n) return true;
    return false;
  };
  if (bad_idx(c->bonds) || bad_idx(c->angles) || bad_idx(c->dihedrals) || bad_idx(c->impropers) ||
      bad_idx(c->excl) || bad_idx(c->cons))
    return og_fail(OG_E_BADARG, "topology atom index out of range");
  return OG_OK;
}

struct SysHost {
  TopoCopy topo;
  std::vector<double> xyz;
  double temperature = 310.0;
  int atom_begin = 0, n_tiles = 0, tile_begin = 0;
};

double deg2rad(double d) { return d * M_PI / 180.0; }

}  // namespace

struct og_engine {
  og_params p{};
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::vector<SysHost> sys;
  bool finalized = false;
  bool forces_valid = false;
  int n_padded = 0, n_tiles = 0;

  // per padded atom
  DVec<double> x, y, z, vx, vy, vz, rx, ry, rz, mass, inv_mass, q, rmin, eps, rmin14, eps14, rho, rho_tilde, srho;
  DVec<double> born_r, born_r64, integral64, e_lj, e_coul, e_gb, e_self;
  DVec<unsigned long long> fx, fy, fz, born_sum;
  DVec<int32_t> atom_sys, local_idx, atom_valid, n_pairs;
  // real atom (systems in order) -> padded index; AoS staging of og_state
  DVec<int32_t> real_map;
  int64_t n_real = 0;
  DVec<double> stage_a, stage_b;
  DVec<int64_t> stage_f;
  DVec<float> pq, lj, gb;  // tile-SoA, 4 columns per 32-atom tile
  DVec<double4> origin;
  DVec<ogk::SysState> sys_state;
  // pair work
  DVec<ogk::PairWork> work;
  DVec<int32_t> jlist, mask_begin;
  DVec<ogk::TileMaskRef> mask_refs;
  DVec<uint32_t> mask_ex, mask_14;
  DVec<int32_t> excl_row, excl_col;
  DVec<int8_t> excl_kind;
  DVec<int4> near;
  // Host side of the exclusion tables, kept so that an append
  // (og_engine_append_atoms) adds only the new exclusions' bits: mask block
  // of each ordered tile pair, the blocks' words, per-tile block references
  // (sorted by j tile) and their CSR, per-atom exclusion rows and their CSR,
  // the unordered near-field block list.
  std::map<std::pair<int, int>, int> mask_of;
  std::vector<uint32_t> h_mex, h_m14;
  std::vector<std::vector<ogk::TileMaskRef>> tile_refs;
  std::vector<int32_t> h_mask_begin;
  std::vector<ogk::TileMaskRef> h_mask_refs;
  std::vector<std::vector<std::pair<int, int8_t>>> excl_rows;
  std::vector<int32_t> h_excl_row, h_excl_col;
  std::vector<int8_t> h_excl_kind;
  std::vector<int4> h_near;
  int n_terms = 0;  // dihedral Fourier terms on the device
  // FP64 energy path: j ranges per i atom and their partial sums
  int e_chunks = 1;
  DVec<double> epart;
  DVec<int32_t> epart_pairs;
  DVec<ogk::PairWork> work_f;   // far-field force: upper-triangle tile pairs
  DVec<int32_t> jlist_f;
  // cutoff mode: i-blocks of the two lists, their culled j lists and ends
  DVec<ogk::CutBlock> cut_b, cut_f;
  DVec<int32_t> jlist_cut_b, jlist_cut_f, seg_end_b, seg_end_f;
  int n_cut_b = 0, n_cut_f = 0;
  int n_work = 0, n_near = 0, n_work_f = 0;
  // how the two pair passes are launched and chunked (og_engine_autotune),
  // and the persistent launches' queue heads (Born, force)
  ogk::PairLaunch born_launch, force_launch;
  int chunk_b = 16, chunk_f = 16;
  DVec<int32_t> pair_queue;
  // device-side replica exchange (og_remd_run): temperature slots, counters
  bool remd_ready = false;
  uint32_t remd_round = 0;
  DVec<int32_t> remd_slot, remd_begin, remd_count;
  DVec<double> remd_temps, remd_total, remd_vscale;
  DVec<long long> remd_attempts, remd_accepts;
  // bonded
  DVec<int2> bond_atoms, dih_terms;
  DVec<int4> angle_atoms, dih_atoms, imp_atoms;
  DVec<double> bond_k, bond_r0, angle_k, angle_t0, term_k, term_delta, imp_k, imp_psi0, bonded_e;
  DVec<int32_t> term_n;
  int n_bonds = 0, n_angles = 0, n_dih = 0, n_imp = 0;
  // SHAKE
  DVec<int32_t> cl_start, cl_sys;
  DVec<int2> cons_atoms;
  DVec<double> cons_d2;
  int n_clusters = 0;
  // reductions
  DVec<int32_t> seg_begin, seg_end;  // [atoms per sys | bonds | angles | dihedrals | impropers], 5*n_sys
  DVec<double> seg_out;
  DVec<int32_t> clamp_count, error_flag, sys_nonfinite;
  // SASA: per padded atom radius (vdW + probe) and surface tension, the
  // atoms with non-zero tension (force / energy tasks) and all real atoms
  // (area queries), per-system tile ranges, component probes, test points.
  DVec<double> sasa_r, sasa_gamma, sasa_area, sasa_energy, sasa_probes, sr_dots;
  DVec<int32_t> sasa_tasks, sasa_all, probe_begin;
  DVec<int16_t> probe_adj;
  DVec<int2> sys_tiles;
  DVec<ogk::SasaArcTerm> sasa_arc_terms;
  DVec<ogk::SasaVertexTerm> sasa_vertex_terms;
  DVec<int32_t> sasa_counts, sasa_overflow;
  int sasa_term_cap = 0;
  int n_sasa_tasks = 0, n_sasa_all = 0, n_sr_dots = 0;
  // learned Born radii: descriptor class per atom, network input, Coulomb-
  // field radii, two hidden-layer buffers, parameters; judge state
  DVec<int32_t> lgb_class;
  DVec<float> lgb_x, lgb_ha, lgb_hb, lgb_params;
  DVec<double> lgb_rcfa, lgb_part;
  DVec<unsigned long long> lgb_fx, lgb_fy, lgb_fz;
  bool lgb_params_set = false, lgb_active = false;
  // the network as three GEMM launches + head (OG_LGB_UNFUSED=1) instead of
  // the fused kernel; both give the same radii
  bool lgb_unfused = false;
  int n_sm = 148;
  int lgb_judge_interval = 500, lgb_judged = 0;
  double lgb_tol = 1e-3, lgb_last_err = -1.0;
  int64_t lgb_since_judge = 0;
  // external potential: the cotranslation exit tunnel
  bool tunnel_on = false;
  ogk::TunnelParams tunnel{};
  double sasa_rmax = 0.0;
  // graph
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  // profiling
  bool profile = false;
  std::map<std::string, std::pair<double, long long>> prof;
  std::vector<std::string> prof_names;

  ~og_engine() {
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    if (graph) cudaGraphDestroy(graph);
    if (own_stream && stream) cudaStreamDestroy(stream);
    for (cudaStream_t* q : {&side, &hi})
      if (*q) {
        cudaStreamSynchronize(*q);
        cudaStreamDestroy(*q);
      }
    for (cudaEvent_t ev : {ev_fork, ev_join, ev_join_hi})
      if (ev) cudaEventDestroy(ev);
  }

  // The surface term runs on an internal side stream, forked after the
  // positions are packed and joined before anything reads the forces, so
  // its FP64, latency-bound kernels overlap the FP32 pair kernels (both add
  // into the fixed-point accumulators with atomics, so the result does not
  // depend on the interleaving).  Inside a graph capture the fork and join
  // become graph edges.
  // The pair kernels go to a high-priority internal stream and the surface
  // term to a low-priority one; in eager launches (judge, single force
  // evaluations) the block scheduler then places pair blocks first.
  cudaStream_t side = nullptr, hi = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_join_hi = nullptr;
  cudaError_t ensure_side() {
    if (side) return cudaSuccess;
    int least = 0, greatest = 0;
    cudaError_t e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
    if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&side, cudaStreamNonBlocking, least);
    if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&hi, cudaStreamNonBlocking, greatest);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev_join_hi, cudaEventDisableTiming);
    return e;
  }

  ogk::AtomArrays atoms() {
    ogk::AtomArrays a{};
    a.n_padded = n_padded;
    a.x = x.p; a.y = y.p; a.z = z.p;
    a.vx = vx.p; a.vy = vy.p; a.vz = vz.p;
    a.rx = rx.p; a.ry = ry.p; a.rz = rz.p;
    a.fx = fx.p; a.fy = fy.p; a.fz = fz.p;
    a.born_sum = born_sum.p;
    a.mass = mass.p;
    a.atom_sys = atom_sys.p;
    a.local_idx = local_idx.p;
    a.q = q.p;
    a.rho = rho.p;
    a.rho_tilde = rho_tilde.p;
    a.srho = srho.p;
    a.pq = pq.p;
    a.gb = gb.p;
    a.origin = origin.p;
    a.born_r = born_r.p;
    a.sys = sys_state.p;
    a.sys_nonfinite = sys_nonfinite.p;
    return a;
  }

  ogk::PairArgs pair_args() {
    ogk::PairArgs a{};
    a.pq = pq.p; a.lj = lj.p; a.gb = gb.p; a.origin = origin.p; a.atom_valid = atom_valid.p;
    a.work = work.p; a.n_work = n_work; a.jlist = jlist.p;
    a.mask_begin = mask_begin.p; a.mask_refs = mask_refs.p; a.mask_ex = mask_ex.p; a.mask_14 = mask_14.p;
    a.fx = fx.p; a.fy = fy.p; a.fz = fz.p; a.born_sum = born_sum.p;
    auto c2 = [](double c) { return no_cutoff(c) ? INFINITY : static_cast<float>(c * c); };
    a.nb_c2 = c2(p.nb_cutoff);
    a.gb_c2 = c2(p.gb_force_cutoff);
    a.born_c2 = c2(p.born_cutoff);
    a.inv_rc3 = no_cutoff(p.nb_cutoff) ? 0.0f
                                       : static_cast<float>(1.0 / (p.nb_cutoff * p.nb_cutoff * p.nb_cutoff));
    a.coul_kj = static_cast<float>(ogk::kCoulomb * ogk::kKcalToKj);
    a.lj_kj12 = static_cast<float>(12.0 * ogk::kKcalToKj);
    a.gb_pref_kj = static_cast<float>((1.0 - 1.0 / ogk::kEpsWater) * ogk::kCoulomb * ogk::kKcalToKj);
    a.error_flag = error_flag.p;
    a.queue = pair_queue.p;
    a.atom_sys = atom_sys.p;
    a.sys_nonfinite = sys_nonfinite.p;
    a.x64 = x.p; a.y64 = y.p; a.z64 = z.p; a.q64 = q.p;
    a.rmin64 = rmin.p; a.eps64 = eps.p; a.rmin14_64 = rmin14.p; a.eps14_64 = eps14.p;
    a.born_r64 = born_r.p;
    auto c2d = [](double c) { return no_cutoff(c) ? static_cast<double>(INFINITY) : c * c; };
    a.nb_c2_64 = c2d(p.nb_cutoff);
    a.gb_c2_64 = c2d(p.gb_force_cutoff);
    a.inv_rc3_64 = no_cutoff(p.nb_cutoff) ? 0.0 : 1.0 / (p.nb_cutoff * p.nb_cutoff * p.nb_cutoff);
    return a;
  }

  ogk::BondedArgs bonded_args() {
    ogk::BondedArgs a{};
    a.x = x.p; a.y = y.p; a.z = z.p;
    a.n_bonds = n_bonds; a.n_angles = n_angles; a.n_dihedrals = n_dih; a.n_impropers = n_imp;
    a.bond_atoms = bond_atoms.p; a.bond_k = bond_k.p; a.bond_r0 = bond_r0.p;
    a.angle_atoms = angle_atoms.p; a.angle_k = angle_k.p; a.angle_t0 = angle_t0.p;
    a.dih_atoms = dih_atoms.p; a.dih_terms = dih_terms.p;
    a.term_k = term_k.p; a.term_n = term_n.p; a.term_delta = term_delta.p;
    a.imp_atoms = imp_atoms.p; a.imp_k = imp_k.p; a.imp_psi0 = imp_psi0.p;
    a.fx = fx.p; a.fy = fy.p; a.fz = fz.p;
    a.energy = bonded_e.p;
    a.atom_sys = atom_sys.p;
    a.sys_nonfinite = sys_nonfinite.p;
    return a;
  }

  ogk::SasaArgs sasa_args(bool all_atoms) {
    ogk::SasaArgs a{};
    a.x = x.p; a.y = y.p; a.z = z.p;
    a.radius = sasa_r.p;
    a.gamma = sasa_gamma.p;
    a.tasks = all_atoms ? sasa_all.p : sasa_tasks.p;
    a.n_tasks = all_atoms ? n_sasa_all : n_sasa_tasks;
    a.atom_sys = atom_sys.p;
    a.sys_tiles = sys_tiles.p;
    a.origin = origin.p;
    a.r_max = sasa_rmax;
    a.fx = fx.p; a.fy = fy.p; a.fz = fz.p;
    a.area = sasa_area.p;
    a.energy = sasa_energy.p;
    a.probes = sasa_probes.p;
    a.probe_adj_begin = probe_begin.p;
    a.probe_adj = probe_adj.p;
    a.sys = sys_state.p;
    a.arc_terms = sasa_arc_terms.p;
    a.vertex_terms = sasa_vertex_terms.p;
    a.counts = sasa_counts.p;
    a.term_cap = sasa_term_cap;
    a.overflow = sasa_overflow.p;
    a.overflow_cap = static_cast<int32_t>(sasa_overflow.n);
    return a;
  }

  ogk::StepArgs step_args() {
    ogk::StepArgs s{};
    s.at = atoms();
    s.half_dt = 0.5 * p.dt_fs;
    s.alpha = std::exp(-p.friction_ps_inv * p.dt_fs * 1.0e-3);
    s.seed_lo = static_cast<uint32_t>(p.seed);
    s.seed_hi = static_cast<uint32_t>(p.seed >> 32);
    s.use_shake = (p.constrain_h_bonds && n_clusters > 0) ? 1 : 0;
    return s;
  }

  ogk::ShakeArgs shake_args() {
    ogk::ShakeArgs a{};
    a.x = x.p; a.y = y.p; a.z = z.p;
    a.rx = rx.p; a.ry = ry.p; a.rz = rz.p;
    a.inv_mass = inv_mass.p;
    a.n_clusters = n_clusters;
    a.cluster_start = cl_start.p;
    a.cluster_sys = cl_sys.p;
    a.cons_atoms = cons_atoms.p;
    a.cons_d2 = cons_d2.p;
    a.tol_sq = p.shake_tol_sq > 0.0 ? p.shake_tol_sq : 1e-6;
    a.max_iters = p.shake_max_iters > 0 ? p.shake_max_iters : 64;
    a.sys = sys_state.p;
    return a;
  }

  // --- profiling helpers (used only outside graph capture)
  struct Timer {
    og_engine* e;
    const char* name;
    cudaStream_t s;
    cudaEvent_t a = nullptr, b = nullptr;
    Timer(og_engine* eng, const char* n, cudaStream_t on = nullptr) : e(eng), name(n), s(on ? on : eng->stream) {
      if (!e->profile) return;
      cudaEventCreate(&a);
      cudaEventCreate(&b);
      cudaEventRecord(a, s);
    }
    ~Timer() {
      if (!e->profile) return;
      cudaEventRecord(b, s);
      cudaEventSynchronize(b);
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, a, b);
      auto& slot = e->prof[name];
      slot.first += ms;
      slot.second += 1;
      cudaEventDestroy(a);
      cudaEventDestroy(b);
    }
  };

  bool lgb_on() const { return p.born_mode == 1 && lgb_active; }

  ogk::LgbDescArgs lgb_desc_args() {
    ogk::LgbDescArgs a{};
    a.x = x.p; a.y = y.p; a.z = z.p;
    a.atom_sys = atom_sys.p;
    a.klass = lgb_class.p;
    a.rho = rho.p;
    a.rho_tilde = rho_tilde.p;
    a.srho = srho.p;
    a.sys_tiles = sys_tiles.p;
    a.origin = origin.p;
    a.n_padded = n_padded;
    a.xin = lgb_x.p;
    a.r_cfa = lgb_rcfa.p;
    return a;
  }

  // One tensor-core layer of the radius network over every padded atom:
  // out = SiLU(in W^T + b) (the epilogue writes z, then SiLU(z), in place).
  void lgb_layer(const float* in, int k_in, int w_off, int b_off, float* out) {
    ogk::TcGemmArgs g{};
    g.a = in; g.a_sm = k_in; g.a_sk = 1;
    g.b = lgb_params.p + w_off; g.b_sn = k_in; g.b_sk = 1;
    g.c = out; g.c_sm = ogk::kLgbHidden; g.c_sn = 1;
    g.m = n_padded; g.n = ogk::kLgbHidden; g.k = k_in;
    g.bias = lgb_params.p + b_off;
    g.c_act = out;
    g.error_flag = error_flag.p;
    ogk::launch_tc_gemm(g, 1, nullptr, stream);
  }

  // Radii from the network: descriptors, three hidden layers, head.
  void enqueue_learned_radii() {
    {
      Timer t(this, "lgb_descriptors");
      ogk::launch_lgb_descriptors(lgb_desc_args(), stream);
    }
    {
      Timer t(this, "lgb_network");
      if (lgb_unfused) {
        lgb_layer(lgb_x.p, ogk::kLgbIn, ogk::kLgbOffW1, ogk::kLgbOffB1, lgb_ha.p);
        lgb_layer(lgb_ha.p, ogk::kLgbHidden, ogk::kLgbOffW2, ogk::kLgbOffB2, lgb_hb.p);
        lgb_layer(lgb_hb.p, ogk::kLgbHidden, ogk::kLgbOffW3, ogk::kLgbOffB3, lgb_ha.p);
        ogk::launch_lgb_radii(atoms(), lgb_ha.p, lgb_x.p, lgb_params.p, lgb_rcfa.p, stream);
      } else {
        ogk::launch_lgb_mlp_radii(atoms(), lgb_x.p, lgb_params.p, lgb_rcfa.p, error_flag.p, n_sm, stream);
      }
    }
  }

  // Force evaluation on the device (positions already packed and
  // accumulators zeroed): Born radii (descreening pass, or the learned
  // network), fused pair force, bonded terms, surface term.
  void enqueue_forces() {
    ogk::PairArgs pa = pair_args();
    ogk::AtomArrays at = atoms();
    // the surface term on the side stream (profiling times kernels one by
    // one, on the main stream)
    const bool sasa_forked = p.include_sasa && !profile && ensure_side() == cudaSuccess;
    const cudaStream_t main_stream = stream;
    if (sasa_forked) {
      cudaEventRecord(ev_fork, stream);
      cudaStreamWaitEvent(side, ev_fork, 0);
      cudaStreamWaitEvent(hi, ev_fork, 0);
      ogk::launch_sasa_forces(sasa_args(false), side);
      cudaEventRecord(ev_join, side);
      stream = hi;  // the pair kernels below
    }
    if (lgb_on()) {
      enqueue_learned_radii();
    } else {
      {
        Timer t(this, "born_pass");
        ogk::PairArgs pb = pa;
        if (!no_cutoff(p.born_cutoff)) {
          ogk::launch_cut_lists(cut_b.p, n_cut_b, jlist.p, origin.p, p.born_cutoff, jlist_cut_b.p, seg_end_b.p,
                                stream);
          pb.jlist = jlist_cut_b.p;
          pb.seg_end = seg_end_b.p;
        }
        ogk::launch_born_pass(pb, born_launch, stream);
      }
      {
        Timer t(this, "born_finalize");
        ogk::launch_born_finalize(at, nullptr, born_r.p, true, nullptr, stream);
      }
    }
    {
      Timer t(this, "force_pass");
      ogk::PairArgs pf = pa;
      pf.work = work_f.p;
      pf.n_work = n_work_f;
      pf.jlist = jlist_f.p;
      pf.queue = pair_queue.p + 1;
      if (!no_cutoff(p.nb_cutoff) && !no_cutoff(p.gb_force_cutoff)) {
        ogk::launch_cut_lists(cut_f.p, n_cut_f, jlist_f.p, origin.p, std::max(p.nb_cutoff, p.gb_force_cutoff),
                              jlist_cut_f.p, seg_end_f.p, stream);
        pf.jlist = jlist_cut_f.p;
        pf.seg_end = seg_end_f.p;
      }
      ogk::launch_force_pass(pf, force_launch, stream);
    }
    {
      Timer t(this, "near_force64");
      ogk::launch_near_force64(pa, near.p, n_near, stream);
    }
    {
      Timer t(this, "bonded");
      ogk::launch_bonded_forces(bonded_args(), stream);
    }
    if (sasa_forked) {
      cudaEventRecord(ev_join_hi, hi);
      stream = main_stream;
      cudaStreamWaitEvent(stream, ev_join_hi, 0);
      cudaStreamWaitEvent(stream, ev_join, 0);
    } else if (p.include_sasa) {
      Timer t(this, "sasa");
      ogk::launch_sasa_forces(sasa_args(false), stream);
    }
    if (tunnel_on) {
      Timer t(this, "tunnel");
      ogk::launch_tunnel(atoms(), tunnel, stream);
    }
  }

  void enqueue_step() {
    ogk::StepArgs sa = step_args();
    {
      Timer t(this, "step_pre");
      ogk::launch_step_pre(sa, stream);
    }
    if (sa.use_shake) {
      Timer t(this, "shake");
      ogk::launch_shake(shake_args(), stream);
    }
    {
      Timer t(this, "step_mid");
      ogk::launch_step_mid(sa, stream);
    }
    if (sa.use_shake) {
      Timer t(this, "shake");
      ogk::launch_shake(shake_args(), stream);
    }
    {
      Timer t(this, "step_post");
      ogk::launch_step_post(sa, stream);
    }
    enqueue_forces();
    {
      Timer t(this, "step_end");
      ogk::launch_step_end(sa, stream);
    }
  }
};

namespace {

og_status check_ready(const og_engine* e) {
  if (!e) return og_fail(OG_E_BADARG, "null engine");
  if (!e->finalized) return og_fail(OG_E_STATE, "engine not finalized");
  return OG_OK;
}

og_status check_sys(const og_engine* e, int32_t s) {
  og_status st = check_ready(e);
  if (st != OG_OK) return st;
  if (s < 0 || s >= static_cast<int32_t>(e->sys.size())) return og_fail(OG_E_BADARG, "system index out of range");
  return OG_OK;
}

og_status launch_check(const char* what) {
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return cuda_fail(err, what);
  return OG_OK;
}

og_status read_status(og_engine* e, std::vector<ogk::SysState>* out) {
  out->resize(e->sys.size());
  OG_CUDA(cudaMemcpyAsync(out->data(), e->sys_state.p, sizeof(ogk::SysState) * e->sys.size(),
                          cudaMemcpyDeviceToHost, e->stream));
  int32_t err_flag = 0;
  OG_CUDA(cudaMemcpyAsync(&err_flag, e->error_flag.p, sizeof(int32_t), cudaMemcpyDeviceToHost, e->stream));
  OG_CUDA(cudaStreamSynchronize(e->stream));
  if (err_flag & ogk::kStatusTimeout) return og_fail(OG_E_TIMEOUT, "a pair-kernel pipeline wait timed out");
  for (const auto& s : *out)
    if (s.status & ogk::kStatusSasaOverflow)
      return og_fail(OG_E_UNSUPPORTED, "an atom's SASA arrangement exceeds the kernels' largest capacity (254 "
                                       "caps, 254 transitions per circle, 128 arcs, or the term buffers); its "
                                       "surface term was not evaluated");
  return OG_OK;
}

// Fibonacci test points of the Shrake-Rupley sampler (sasa.rs:182-197).
std::vector<double> sr_dot_table(int n) {
  std::vector<double> d(3 * static_cast<size_t>(n));
  const double phi = M_PI * (std::sqrt(3.0) + 1.0);
  for (int k = 0; k < n; ++k) {
    const double yy = 1.0 - 2.0 * k / (n - 1.0);
    const double rr = std::sqrt(1.0 - yy * yy);
    d[3 * k] = std::cos(phi * k) * rr;
    d[3 * k + 1] = yy;
    d[3 * k + 2] = std::sin(phi * k) * rr;
  }
  return d;
}

// Per-atom areas of every real atom into e->sasa_area (method 0 PowerSasa,
// 1 Shrake-Rupley with `dots`), from the current positions.
og_status sasa_areas_all(og_engine* e, int method, const double* dots, int n_dots) {
  cudaStream_t st = e->stream;
  OG_CUDA(cudaMemsetAsync(e->sasa_area.p, 0, sizeof(double) * e->n_padded, st));
  OG_CUDA(cudaMemsetAsync(e->sasa_energy.p, 0, sizeof(double) * e->n_padded, st));
  ogk::launch_pack(e->atoms(), false, st);
  if (method == 0) ogk::launch_sasa_areas(e->sasa_args(true), st);
  else ogk::launch_shrake_rupley(e->sasa_args(true), dots, n_dots, st);
  og_status s = launch_check("SASA area kernel");
  if (s != OG_OK) return s;
  std::vector<ogk::SysState> hs;
  return read_status(e, &hs);
}

// xoshiro256++ / SplitMix64 / Box-Muller exactly as dynamics/src/rng.rs.
struct Xoshiro {
  uint64_t s[4];
  bool has_spare = false;
  double spare = 0.0;
  explicit Xoshiro(uint64_t seed) {
    uint64_t sm = seed;
    for (int k = 0; k < 4; ++k) {
      sm += 0x9e3779b97f4a7c15ULL;
      uint64_t z = sm;
      z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
      z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
      s[k] = z ^ (z >> 31);
    }
  }
  static uint64_t rotl(uint64_t v, int k) { return (v << k) | (v >> (64 - k)); }
  uint64_t next_u64() {
    uint64_t result = rotl(s[0] + s[3], 23) + s[0];
    uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return result;
  }
  double next_f64() { return static_cast<double>(next_u64() >> 11) * (1.0 / static_cast<double>(1ULL << 53)); }
  double gaussian() {
    if (has_spare) {
      has_spare = false;
      return spare;
    }
    double u1 = next_f64();
    while (u1 <= 0.0) u1 = next_f64();
    double u2 = next_f64();
    double r = std::sqrt(-2.0 * std::log(u1));
    double th = 2.0 * M_PI * u2;
    spare = r * std::sin(th);
    has_spare = true;
    return r * std::cos(th);
  }
};

template <class T>
og_status copy_sys_range(og_engine* e, const DVec<T>& v, int s, T* host) {
  const SysHost& sh = e->sys[s];
  OG_CUDA(cudaMemcpyAsync(host, v.p + sh.atom_begin, sizeof(T) * sh.topo.n, cudaMemcpyDeviceToHost, e->stream));
  return OG_OK;
}

// Interleaved xyz <-> SoA device arrays of one system.
og_status get_xyz(og_engine* e, int s, const DVec<double>& a, const DVec<double>& b, const DVec<double>& c,
                  double* out) {
  const int n = e->sys[s].topo.n;
  std::vector<double> hx(n), hy(n), hz(n);
  og_status st;
  if ((st = copy_sys_range(e, a, s, hx.data())) != OG_OK) return st;
  if ((st = copy_sys_range(e, b, s, hy.data())) != OG_OK) return st;
  if ((st = copy_sys_range(e, c, s, hz.data())) != OG_OK) return st;
  OG_CUDA(cudaStreamSynchronize(e->stream));
  for (int i = 0; i < n; ++i) {
    out[3 * i] = hx[i];
    out[3 * i + 1] = hy[i];
    out[3 * i + 2] = hz[i];
  }
  return OG_OK;
}

og_status set_xyz(og_engine* e, int s, DVec<double>& a, DVec<double>& b, DVec<double>& c, const double* in) {
  const SysHost& sh = e->sys[s];
  const int n = sh.topo.n;
  std::vector<double> hx(n), hy(n), hz(n);
  for (int i = 0; i < n; ++i) {
    hx[i] = in[3 * i];
    hy[i] = in[3 * i + 1];
    hz[i] = in[3 * i + 2];
  }
  OG_CUDA(cudaMemcpyAsync(a.p + sh.atom_begin, hx.data(), sizeof(double) * n, cudaMemcpyHostToDevice, e->stream));
  OG_CUDA(cudaMemcpyAsync(b.p + sh.atom_begin, hy.data(), sizeof(double) * n, cudaMemcpyHostToDevice, e->stream));
  OG_CUDA(cudaMemcpyAsync(c.p + sh.atom_begin, hz.data(), sizeof(double) * n, cudaMemcpyHostToDevice, e->stream));
  OG_CUDA(cudaStreamSynchronize(e->stream));
  return OG_OK;
}

// Pair work (Newton-3 layout): i-blocks of W consecutive tiles (W from the
// pass's launch shape) against the tiles from the block's first tile on
// (Born pass: the block's own diagonal included) or after it (far-field
// force pass), cut into chunks of at most `chunk` j-tiles and ordered
// longest first; plus the i-blocks of cutoff mode's culled lists.
og_status build_pass_list(og_engine* e, int first_offset, int W, int chunk, DVec<ogk::PairWork>* work,
                          int* n_work, DVec<int32_t>* jlist, DVec<ogk::CutBlock>* cut, int* n_cut,
                          DVec<int32_t>* jlist_cut, DVec<int32_t>* seg_end, cudaStream_t st) {
  std::vector<int32_t> hj;
  std::vector<ogk::PairWork> hw;
  std::vector<ogk::CutBlock> hc;
  for (const auto& s : e->sys) {
    for (int t0 = 0; t0 < s.n_tiles; t0 += W) {
      const int jb = static_cast<int>(hj.size());
      for (int t = t0 + first_offset; t < s.n_tiles; ++t) hj.push_back(s.tile_begin + t);
      const int je = static_cast<int>(hj.size());
      hc.push_back(ogk::CutBlock{s.tile_begin + t0, std::min(W, s.n_tiles - t0), jb, je});
      for (int j0 = jb; j0 < je; j0 += chunk)
        hw.push_back(ogk::PairWork{s.tile_begin + t0, std::min(W, s.n_tiles - t0), j0, std::min(je, j0 + chunk)});
    }
  }
  std::stable_sort(hw.begin(), hw.end(), [](const ogk::PairWork& a, const ogk::PairWork& b) {
    return (a.j_end - a.j_begin) > (b.j_end - b.j_begin);
  });
  *n_cut = static_cast<int>(hc.size());
  OG_CUDA(cut->upload(hc, st));
  OG_CUDA(jlist_cut->alloc(std::max<size_t>(hj.size(), 1)));
  OG_CUDA(seg_end->alloc(std::max(e->n_tiles, 1)));
  *n_work = static_cast<int>(hw.size());
  OG_CUDA(work->upload(hw, st));
  OG_CUDA(jlist->upload(hj, st));
  return OG_OK;
}

og_status build_pair_lists(og_engine* e, cudaStream_t st) {
  og_status s = build_pass_list(e, 0, ogk::pair_shape_tiles(e->born_launch.shape), e->chunk_b, &e->work, &e->n_work,
                                &e->jlist, &e->cut_b, &e->n_cut_b, &e->jlist_cut_b, &e->seg_end_b, st);
  if (s != OG_OK) return s;
  return build_pass_list(e, 1, ogk::pair_shape_tiles(e->force_launch.shape), e->chunk_f, &e->work_f, &e->n_work_f,
                         &e->jlist_f, &e->cut_f, &e->n_cut_f, &e->jlist_cut_f, &e->seg_end_f, st);
}

template <class T>
cudaError_t put(DVec<T>& d, size_t at, const std::vector<T>& h, cudaStream_t st) {
  if (h.empty()) return cudaSuccess;
  return cudaMemcpyAsync(d.p + at, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, st);
}

// Appends h to the device array (grown to n + h.size() elements).
template <class T>
cudaError_t append(DVec<T>& d, const std::vector<T>& h, cudaStream_t st) {
  const size_t at = d.n;
  cudaError_t e = d.grow(at + h.size(), st);
  if (e != cudaSuccess || h.empty()) return e;
  return cudaMemcpyAsync(d.p + at, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, st);
}

// The system owning padded atom i (-1 for padding past the last system).
int system_of(const og_engine* e, int i) {
  auto it = std::upper_bound(e->sys.begin(), e->sys.end(), i,
                             [](int v, const SysHost& s) { return v < s.atom_begin; });
  if (it == e->sys.begin()) return -1;
  const int si = static_cast<int>(it - e->sys.begin()) - 1;
  return i < e->sys[si].atom_begin + e->sys[si].topo.n ? si : -1;
}

// Static per-atom tables of the padded atoms [a0, a1), a0 on a tile
// boundary: force-field parameters, the tile-SoA LJ and GB columns, owner
// system, local index and valid flag, the SASA radius (Bondi vdW + 1.4 A
// probe) and surface tension (0.005 kcal/mol/A^2 on C and S,
// powersasa/mod.rs:27-52, times sasa_gamma_scale, analytical.rs:607-614),
// and the learned-radius descriptor class (C,S -> 0; N,P -> 1; O -> 2;
// H -> 3).  Padding atoms get unit mass, no charge and R = rho~ = 1.  The
// device arrays must hold at least a1 atoms.
og_status fill_atoms(og_engine* e, int a0, int a1, cudaStream_t st) {
  static const double kVdw[6] = {1.20, 1.70, 1.55, 1.52, 1.80, 1.80};
  static const int32_t kClass[6] = {3, 0, 1, 2, 1, 0};
  const double g_cs = 0.005 * ogk::kKcalToKj * e->p.sasa_gamma_scale;
  const size_t m = static_cast<size_t>(a1 - a0);
  std::vector<double> hm(m, 1.0), him(m, 1.0), hq(m, 0.0), hrm(m, 0.0), hep(m, 0.0), hrm14(m, 0.0),
      hep14(m, 0.0), hrho(m, 1.0), hrt(m, 1.0), hsr(m, 0.0), hr(m, 0.0), hg(m, 0.0);
  std::vector<int32_t> hsys(m, -1), hloc(m, 0), hvalid(m, 0), hcls(m, 0);
  std::vector<float> hlj(4 * m, 0.0f), hgb(4 * m);
  for (size_t r = 0; r < m; ++r) {
    const int i = a0 + static_cast<int>(r);
    const int si = system_of(e, i);
    if (si >= 0) {
      const TopoCopy& t = e->sys[si].topo;
      const int k = i - e->sys[si].atom_begin;
      const int el = t.element[k];
      if (el < 0 || el > 5) return og_fail(OG_E_BADARG, "element code out of range");
      hm[r] = t.mass[k];
      him[r] = 1.0 / t.mass[k];
      hq[r] = t.charge[k];
      hrm[r] = t.rmin[k];
      hep[r] = t.eps[k];
      hrm14[r] = t.rmin14[k];
      hep14[r] = t.eps14[k];
      hrho[r] = t.rho[k];
      hrt[r] = t.rho[k] - ogk::kObcOffset;
      hsr[r] = t.scale[k] * hrt[r];
      hsys[r] = si;
      hloc[r] = k;
      hvalid[r] = 1;
      hr[r] = kVdw[el] + 1.4;
      hg[r] = (el == 1 || el == 5) ? g_cs : 0.0;
      hcls[r] = kClass[el];
    }
    const int ri = static_cast<int>(r);
    hlj[ogk::soa_index(ri, 0)] = static_cast<float>(hrm[r]);
    hlj[ogk::soa_index(ri, 1)] = static_cast<float>(std::sqrt(hep[r]));
    hlj[ogk::soa_index(ri, 2)] = static_cast<float>(hrm14[r]);
    hlj[ogk::soa_index(ri, 3)] = static_cast<float>(std::sqrt(hep14[r]));
    // The Born pass reads rho~ and s*rho~ before the first radii exist, so
    // the gb columns start out fully defined (R = rho~ until then).
    const bool real = si >= 0;
    hgb[ogk::soa_index(ri, 0)] = real ? static_cast<float>(hrt[r]) : 1.0f;
    hgb[ogk::soa_index(ri, 1)] = real ? static_cast<float>(1.0 / hrt[r]) : 1.0f;
    hgb[ogk::soa_index(ri, 2)] = real ? static_cast<float>(hrt[r]) : 1.0f;
    hgb[ogk::soa_index(ri, 3)] = real ? static_cast<float>(hsr[r]) : 0.0f;
  }
  OG_CUDA(put(e->mass, a0, hm, st)); OG_CUDA(put(e->inv_mass, a0, him, st)); OG_CUDA(put(e->q, a0, hq, st));
  OG_CUDA(put(e->rmin, a0, hrm, st)); OG_CUDA(put(e->eps, a0, hep, st));
  OG_CUDA(put(e->rmin14, a0, hrm14, st)); OG_CUDA(put(e->eps14, a0, hep14, st));
  OG_CUDA(put(e->rho, a0, hrho, st)); OG_CUDA(put(e->rho_tilde, a0, hrt, st)); OG_CUDA(put(e->srho, a0, hsr, st));
  OG_CUDA(put(e->atom_sys, a0, hsys, st)); OG_CUDA(put(e->local_idx, a0, hloc, st));
  OG_CUDA(put(e->atom_valid, a0, hvalid, st));
  OG_CUDA(put(e->lj, 4 * static_cast<size_t>(a0), hlj, st));
  OG_CUDA(put(e->gb, 4 * static_cast<size_t>(a0), hgb, st));
  OG_CUDA(put(e->sasa_r, a0, hr, st)); OG_CUDA(put(e->sasa_gamma, a0, hg, st));
  OG_CUDA(put(e->lgb_class, a0, hcls, st));
  for (double v : hr) e->sasa_rmax = std::max(e->sasa_rmax, v);
  return OG_OK;
}

// Positions of the padded atoms [a0, a1) from the systems' host copies
// (0 for padding); velocities and SHAKE reference positions zero.
og_status fill_positions(og_engine* e, int a0, int a1, cudaStream_t st) {
  const size_t m = static_cast<size_t>(a1 - a0);
  std::vector<double> hx(m, 0.0), hy(m, 0.0), hz(m, 0.0), zeros(m, 0.0);
  for (size_t r = 0; r < m; ++r) {
    const int i = a0 + static_cast<int>(r);
    const int si = system_of(e, i);
    if (si < 0) continue;
    const int k = i - e->sys[si].atom_begin;
    hx[r] = e->sys[si].xyz[3 * k];
    hy[r] = e->sys[si].xyz[3 * k + 1];
    hz[r] = e->sys[si].xyz[3 * k + 2];
  }
  OG_CUDA(put(e->x, a0, hx, st)); OG_CUDA(put(e->y, a0, hy, st)); OG_CUDA(put(e->z, a0, hz, st));
  for (auto* v : {&e->vx, &e->vy, &e->vz, &e->rx, &e->ry, &e->rz}) OG_CUDA(put(*v, a0, zeros, st));
  return OG_OK;
}

// SASA task lists of system si's atoms [k0, k1): atoms with non-zero
// tension (force and energy tasks) and every real atom (area queries).
void sasa_lists(const og_engine* e, int si, int k0, int k1, std::vector<int32_t>* tasks,
                std::vector<int32_t>* all) {
  const SysHost& s = e->sys[si];
  for (int k = k0; k < k1; ++k) {
    const int el = s.topo.element[k];
    all->push_back(s.atom_begin + k);
    if (el == 1 || el == 5) tasks->push_back(s.atom_begin + k);
  }
}

// ---- exclusion tables.  One 32-word block per ordered tile pair holding an
// exclusion (bit c of word a: atoms a, c excluded; 1-4 pairs in the second
// array), each tile's blocks referenced in j-tile order; per-atom exclusion
// rows for the FP64 paths; the unordered block list of the near field.

// The block of (ti, tj), made (and referenced) when missing; *t_min takes
// the lowest tile whose reference list changed.
int mask_block(og_engine* e, int ti, int tj, int* t_min) {
  auto it = e->mask_of.find({ti, tj});
  if (it != e->mask_of.end()) return it->second;
  const int b = static_cast<int>(e->mask_of.size());
  e->mask_of[{ti, tj}] = b;
  e->h_mex.resize(static_cast<size_t>(b + 1) * kTile, 0u);
  e->h_m14.resize(static_cast<size_t>(b + 1) * kTile, 0u);
  auto& refs = e->tile_refs[ti];
  auto pos = std::lower_bound(refs.begin(), refs.end(), tj,
                              [](const ogk::TileMaskRef& r, int j) { return r.j_tile < j; });
  refs.insert(pos, ogk::TileMaskRef{tj, b});
  *t_min = std::min(*t_min, ti);
  if (ti <= tj) e->h_near.push_back(make_int4(ti, tj, b, 0));
  return b;
}

// Self pairs of tiles [t0, t1) (every lane of the diagonal block).
void mask_diagonal(og_engine* e, int t0, int t1, int* t_min, std::set<int>* touched) {
  for (int t = t0; t < t1; ++t) {
    const int b = mask_block(e, t, t, t_min);
    for (int l = 0; l < kTile; ++l) e->h_mex[static_cast<size_t>(b) * kTile + l] |= 1u << l;
    touched->insert(b);
  }
}

// Exclusion k of system si (kind 1: excluded, else a scaled 1-4 pair).
void mask_exclusion(og_engine* e, int si, size_t k, int* t_min, int* a_min, std::set<int>* touched) {
  const SysHost& s = e->sys[si];
  const int i = s.atom_begin + s.topo.excl[2 * k], j = s.atom_begin + s.topo.excl[2 * k + 1];
  const int8_t kind = s.topo.excl_kind[k];
  e->excl_rows[i].push_back({j, kind});
  e->excl_rows[j].push_back({i, kind});
  *a_min = std::min(*a_min, std::min(i, j));
  for (int dir = 0; dir < 2; ++dir) {
    const int a = dir ? j : i, c = dir ? i : j;
    const int b = mask_block(e, a / kTile, c / kTile, t_min);
    const size_t w = static_cast<size_t>(b) * kTile + (a % kTile);
    if (kind == 1) e->h_mex[w] |= 1u << (c % kTile);
    else e->h_m14[w] |= 1u << (c % kTile);
    touched->insert(b);
  }
}

// Device copies of the exclusion tables after blocks up to n_blocks_before
// existed on the device: the touched old blocks, the new blocks, the tile
// CSR from tile t_min on, the atom CSR from atom a_min on and the near-field
// blocks past n_near_before.
og_status upload_exclusions(og_engine* e, int n_blocks_before, int t_min, int a_min, int n_near_before,
                            const std::set<int>& touched, cudaStream_t st) {
  const int nt = e->n_tiles, np = e->n_padded;
  // tile CSR
  t_min = std::min(t_min, std::max(static_cast<int>(e->h_mask_begin.size()) - 1, 0));
  if (e->h_mask_begin.empty()) t_min = 0;
  e->h_mask_refs.resize(e->h_mask_begin.empty() ? 0 : e->h_mask_begin[t_min]);
  e->h_mask_begin.resize(t_min);
  for (int t = t_min; t < nt; ++t) {
    e->h_mask_begin.push_back(static_cast<int32_t>(e->h_mask_refs.size()));
    e->h_mask_refs.insert(e->h_mask_refs.end(), e->tile_refs[t].begin(), e->tile_refs[t].end());
  }
  e->h_mask_begin.push_back(static_cast<int32_t>(e->h_mask_refs.size()));
  OG_CUDA(e->mask_begin.upload_tail(e->h_mask_begin, t_min, st));
  OG_CUDA(e->mask_refs.upload_tail(e->h_mask_refs, e->h_mask_begin[t_min], st));
  // blocks
  OG_CUDA(e->mask_ex.upload_tail(e->h_mex, static_cast<size_t>(n_blocks_before) * kTile, st));
  OG_CUDA(e->mask_14.upload_tail(e->h_m14, static_cast<size_t>(n_blocks_before) * kTile, st));
  for (int b : touched)
    if (b < n_blocks_before) {
      const size_t w0 = static_cast<size_t>(b) * kTile, w1 = w0 + kTile;
      OG_CUDA(e->mask_ex.upload_range(e->h_mex, w0, w1, st));
      OG_CUDA(e->mask_14.upload_range(e->h_m14, w0, w1, st));
    }
  e->n_near = static_cast<int>(e->h_near.size());
  OG_CUDA(e->near.upload_tail(e->h_near, n_near_before, st));
  // atom CSR (rows sorted by partner)
  a_min = std::min(a_min, std::max(static_cast<int>(e->h_excl_row.size()) - 1, 0));
  if (e->h_excl_row.empty()) a_min = 0;
  e->h_excl_col.resize(e->h_excl_row.empty() ? 0 : e->h_excl_row[a_min]);
  e->h_excl_kind.resize(e->h_excl_col.size());
  e->h_excl_row.resize(a_min);
  for (int i = a_min; i < np; ++i) {
    auto& r = e->excl_rows[i];
    std::sort(r.begin(), r.end());
    e->h_excl_row.push_back(static_cast<int32_t>(e->h_excl_col.size()));
    for (auto& pr : r) {
      e->h_excl_col.push_back(pr.first);
      e->h_excl_kind.push_back(pr.second);
    }
  }
  e->h_excl_row.push_back(static_cast<int32_t>(e->h_excl_col.size()));
  OG_CUDA(e->excl_row.upload_tail(e->h_excl_row, a_min, st));
  OG_CUDA(e->excl_col.upload_tail(e->h_excl_col, e->h_excl_row[a_min], st));
  OG_CUDA(e->excl_kind.upload_tail(e->h_excl_kind, e->h_excl_row[a_min], st));
  return OG_OK;
}

// ---- bonded terms of system si (global atom indices, angles in radians),
// the terms listed in `sel` of each kind, appended to the device lists.
struct TermSel {
  std::vector<int> bonds, angles, dihedrals, impropers, excl, cons;
  static TermSel all(const TopoCopy& t) {
    TermSel s;
    auto iota = [](std::vector<int>* v, size_t n) {
      v->resize(n);
      for (size_t k = 0; k < n; ++k) (*v)[k] = static_cast<int>(k);
    };
    iota(&s.bonds, t.bond_k.size());
    iota(&s.angles, t.angle_k.size());
    iota(&s.dihedrals, t.dihedrals.size() / 4);
    iota(&s.impropers, t.imp_k.size());
    iota(&s.excl, t.excl_kind.size());
    iota(&s.cons, t.cons_d.size());
    return s;
  }
};

og_status append_bonded(og_engine* e, int si, const TermSel& sel, cudaStream_t st) {
  const TopoCopy& t = e->sys[si].topo;
  const int o = e->sys[si].atom_begin;
  std::vector<int2> hb, hdt;
  std::vector<int4> ha, hd, hi;
  std::vector<double> hbk, hbr, hak, hat, htk, htd, hik, hip;
  std::vector<int32_t> htn;
  for (int k : sel.bonds) {
    hb.push_back(make_int2(o + t.bonds[2 * k], o + t.bonds[2 * k + 1]));
    hbk.push_back(t.bond_k[k]);
    hbr.push_back(t.bond_r0[k]);
  }
  for (int k : sel.angles) {
    ha.push_back(make_int4(o + t.angles[3 * k], o + t.angles[3 * k + 1], o + t.angles[3 * k + 2], 0));
    hak.push_back(t.angle_k[k]);
    hat.push_back(deg2rad(t.angle_t0[k]));
  }
  for (int k : sel.dihedrals) {
    hd.push_back(make_int4(o + t.dihedrals[4 * k], o + t.dihedrals[4 * k + 1], o + t.dihedrals[4 * k + 2],
                           o + t.dihedrals[4 * k + 3]));
    const int base = e->n_terms + static_cast<int>(htk.size());
    for (int m = t.dih_start[k]; m < t.dih_start[k + 1]; ++m) {
      htk.push_back(t.term_k[m]);
      htn.push_back(t.term_n[m]);
      htd.push_back(deg2rad(t.term_delta[m]));
    }
    hdt.push_back(make_int2(base, e->n_terms + static_cast<int>(htk.size())));
  }
  for (int k : sel.impropers) {
    hi.push_back(make_int4(o + t.impropers[4 * k], o + t.impropers[4 * k + 1], o + t.impropers[4 * k + 2],
                           o + t.impropers[4 * k + 3]));
    hik.push_back(t.imp_k[k]);
    hip.push_back(deg2rad(t.imp_psi0[k]));
  }
  OG_CUDA(append(e->bond_atoms, hb, st)); OG_CUDA(append(e->bond_k, hbk, st));
  OG_CUDA(append(e->bond_r0, hbr, st));
  OG_CUDA(append(e->angle_atoms, ha, st)); OG_CUDA(append(e->angle_k, hak, st));
  OG_CUDA(append(e->angle_t0, hat, st));
  OG_CUDA(append(e->dih_atoms, hd, st)); OG_CUDA(append(e->dih_terms, hdt, st));
  OG_CUDA(append(e->term_k, htk, st)); OG_CUDA(append(e->term_n, htn, st));
  OG_CUDA(append(e->term_delta, htd, st));
  OG_CUDA(append(e->imp_atoms, hi, st)); OG_CUDA(append(e->imp_k, hik, st));
  OG_CUDA(append(e->imp_psi0, hip, st));
  e->n_bonds += static_cast<int>(hb.size());
  e->n_angles += static_cast<int>(ha.size());
  e->n_dih += static_cast<int>(hd.size());
  e->n_imp += static_cast<int>(hi.size());
  e->n_terms += static_cast<int>(htk.size());
  return OG_OK;
}

// Reduction segments: [atoms | bonds | angles | dihedrals | impropers] per
// system, the bonded ones as ranges of the bonded energy array (bonds, then
// angles, dihedrals, impropers); every system's terms of one kind are
// contiguous, in system order.
og_status upload_segments(og_engine* e, cudaStream_t st) {
  const int n_sys = static_cast<int>(e->sys.size());
  std::vector<int32_t> sb(5 * n_sys), se(5 * n_sys);
  int ob = 0, oa = e->n_bonds, od = e->n_bonds + e->n_angles, oi = e->n_bonds + e->n_angles + e->n_dih;
  for (int si = 0; si < n_sys; ++si) {
    const SysHost& s = e->sys[si];
    const TopoCopy& t = s.topo;
    sb[si] = s.atom_begin;
    se[si] = s.atom_begin + t.n;
    const int nb = static_cast<int>(t.bond_k.size()), na = static_cast<int>(t.angle_k.size());
    const int nd = static_cast<int>(t.dihedrals.size() / 4), ni = static_cast<int>(t.imp_k.size());
    sb[n_sys + si] = ob; se[n_sys + si] = ob += nb;
    sb[2 * n_sys + si] = oa; se[2 * n_sys + si] = oa += na;
    sb[3 * n_sys + si] = od; se[3 * n_sys + si] = od += nd;
    sb[4 * n_sys + si] = oi; se[4 * n_sys + si] = oi += ni;
  }
  OG_CUDA(e->bonded_e.grow(std::max(1, e->n_bonds + e->n_angles + e->n_dih + e->n_imp), st));
  OG_CUDA(e->seg_begin.upload(sb, st));
  OG_CUDA(e->seg_end.upload(se, st));
  return OG_OK;
}

// SHAKE clusters of system si from its constraints listed in `cons`: each
// cluster is one heavy atom's X-H constraints in constraint order, clusters
// in order of their heavy atom's first constraint.  `taken` holds the heavy
// atoms (system-local) that already have a cluster on the device; a
// constraint on one of those cannot be appended.
og_status append_clusters(og_engine* e, int si, const std::vector<int>& cons, const std::set<int>& taken,
                          cudaStream_t st) {
  const SysHost& s = e->sys[si];
  const TopoCopy& t = s.topo;
  std::map<int, std::vector<int>> by_heavy;
  std::vector<int> order;
  for (int k : cons) {
    const int a = t.cons[2 * k], b = t.cons[2 * k + 1];
    const int heavy = (t.element[a] == 0) ? b : a;
    if (taken.count(heavy)) return og_fail(OG_E_BADARG, "a new constraint joins an existing SHAKE cluster");
    if (by_heavy.find(heavy) == by_heavy.end()) order.push_back(heavy);
    by_heavy[heavy].push_back(k);
  }
  std::vector<int32_t> hcs, hcsys;
  std::vector<int2> hca;
  std::vector<double> hcd;
  const int base = static_cast<int>(e->cons_atoms.n);
  for (int h : order) {
    for (int k : by_heavy[h]) {
      hca.push_back(make_int2(s.atom_begin + t.cons[2 * k], s.atom_begin + t.cons[2 * k + 1]));
      hcd.push_back(t.cons_d[k] * t.cons_d[k]);
    }
    hcs.push_back(base + static_cast<int32_t>(hca.size()));
    hcsys.push_back(si);
  }
  OG_CUDA(append(e->cl_start, hcs, st));
  OG_CUDA(append(e->cl_sys, hcsys, st));
  OG_CUDA(append(e->cons_atoms, hca, st));
  OG_CUDA(append(e->cons_d2, hcd, st));
  e->n_clusters += static_cast<int>(hcsys.size());
  return OG_OK;
}

og_status upload_sys_tiles(og_engine* e, cudaStream_t st) {
  std::vector<int2> hst;
  for (const auto& s : e->sys) hst.push_back(make_int2(s.tile_begin, s.n_tiles));
  OG_CUDA(e->sys_tiles.upload(hst, st));
  return OG_OK;
}

// Scratch of the surface term for the current task counts: the term records
// of one force evaluation (proteins average a few exposed arcs per C/S atom
// and reach 19; 16 per atom on average is the limit, exceeding it is
// reported as a capacity overflow) and the queue of atoms beyond the default
// arrangement capacities (force path and area queries alike).
og_status size_sasa_scratch(og_engine* e, cudaStream_t st) {
  if (e->p.include_sasa) {
    e->sasa_term_cap = 16 * e->n_sasa_tasks + 1024;
    OG_CUDA(e->sasa_arc_terms.grow(e->sasa_term_cap, st));
    OG_CUDA(e->sasa_vertex_terms.grow(e->sasa_term_cap, st));
  }
  OG_CUDA(e->sasa_overflow.grow(std::max(1, std::max(e->n_sasa_all, e->n_sasa_tasks)), st));
  return OG_OK;
}

// Per-atom buffers of the learned-radius network (born_mode 1).
og_status size_lgb_scratch(og_engine* e, cudaStream_t st) {
  const size_t np = static_cast<size_t>(e->n_padded);
  OG_CUDA(e->lgb_x.grow(np * ogk::kLgbIn, st));
  OG_CUDA(e->lgb_rcfa.grow(np, st));
  OG_CUDA(e->lgb_ha.grow(np * ogk::kLgbHidden, st));
  OG_CUDA(e->lgb_hb.grow(np * ogk::kLgbHidden, st));
  for (auto* v : {&e->lgb_fx, &e->lgb_fy, &e->lgb_fz}) OG_CUDA(v->grow(np, st));
  return OG_OK;
}

// Partial-sum buffers of the FP64 energy path for the current layout.
og_status size_energy_scratch(og_engine* e, cudaStream_t st) {
  int max_n = 1;
  for (const auto& s : e->sys) max_n = std::max(max_n, s.topo.n);
  e->e_chunks = ogk::energy_chunks(e->n_padded, max_n, e->n_sm);
  if (e->e_chunks > 1) {
    const size_t m = static_cast<size_t>(e->e_chunks) * e->n_padded;
    OG_CUDA(e->epart.grow(3 * m, st));
    OG_CUDA(e->epart_pairs.grow(m, st));
  }
  return OG_OK;
}

ogk::SysState sys_state_of(const og_engine* e, int si) {
  const SysHost& s = e->sys[si];
  const int ncons = static_cast<int>(s.topo.cons_d.size());
  const double dof = 3.0 * s.topo.n;
  ogk::SysState h{};
  h.temperature = s.temperature;
  h.kbt = ogk::kBoltzmann * s.temperature;
  h.dof_corr = (e->p.constrain_h_bonds && ncons > 0) ? dof / std::max(dof - ncons, 1.0) : 1.0;
  h.atom_begin = s.atom_begin;
  h.n_atoms = s.topo.n;
  return h;
}

og_status finalize_impl(og_engine* e) {
  const int n_sys = static_cast<int>(e->sys.size());
  if (n_sys == 0) return og_fail(OG_E_STATE, "no systems added");
  cudaStream_t st = e->stream;

  // ---- layout
  int atom = 0;
  for (auto& s : e->sys) {
    s.atom_begin = atom;
    s.n_tiles = (s.topo.n + kTile - 1) / kTile;
    s.tile_begin = atom / kTile;
    atom += s.n_tiles * kTile;
  }
  e->n_padded = atom;
  e->n_tiles = atom / kTile;
  const int np = e->n_padded;

  // ---- per-atom arrays
  for (auto* v : {&e->mass, &e->inv_mass, &e->q, &e->rmin, &e->eps, &e->rmin14, &e->eps14, &e->rho, &e->rho_tilde,
                  &e->srho, &e->sasa_r, &e->sasa_gamma, &e->x, &e->y, &e->z, &e->vx, &e->vy, &e->vz, &e->rx,
                  &e->ry, &e->rz})
    OG_CUDA(v->alloc(np));
  for (auto* v : {&e->atom_sys, &e->local_idx, &e->atom_valid, &e->lgb_class}) OG_CUDA(v->alloc(np));
  OG_CUDA(e->lj.alloc(4 * static_cast<size_t>(np)));
  OG_CUDA(e->gb.alloc(4 * static_cast<size_t>(np)));
  {
    og_status fs = fill_atoms(e, 0, np, st);
    if (fs == OG_OK) fs = fill_positions(e, 0, np, st);
    if (fs != OG_OK) return fs;
  }
  {
    std::vector<int32_t> hmap;
    for (const auto& s : e->sys)
      for (int k = 0; k < s.topo.n; ++k) hmap.push_back(s.atom_begin + k);
    e->n_real = static_cast<int64_t>(hmap.size());
    OG_CUDA(e->real_map.upload(hmap, st));
  }
  for (auto* v : {&e->born_r, &e->born_r64, &e->integral64, &e->e_lj, &e->e_coul, &e->e_gb, &e->e_self})
    OG_CUDA(v->alloc(np));
  for (auto* v : {&e->fx, &e->fy, &e->fz, &e->born_sum}) OG_CUDA(v->alloc(np));
  OG_CUDA(e->n_pairs.alloc(np));
  OG_CUDA(e->pq.alloc(4 * static_cast<size_t>(np)));
  OG_CUDA(e->origin.alloc(e->n_tiles));

  // ---- SASA task lists, term records, overflow queue (radius and tension
  // per atom come with the per-atom arrays)
  {
    std::vector<int32_t> htask, hall;
    for (int si = 0; si < n_sys; ++si) sasa_lists(e, si, 0, e->sys[si].topo.n, &htask, &hall);
    e->n_sasa_tasks = static_cast<int>(htask.size());
    e->n_sasa_all = static_cast<int>(hall.size());
    OG_CUDA(e->sasa_tasks.upload(htask, st));
    OG_CUDA(e->sasa_all.upload(hall, st));
    og_status ts = upload_sys_tiles(e, st);
    if (ts != OG_OK) return ts;
    OG_CUDA(e->sasa_area.alloc(np));
    OG_CUDA(e->sasa_energy.alloc(np));
    OG_CUDA(e->sasa_counts.alloc(4));
    if ((ts = size_sasa_scratch(e, st)) != OG_OK) return ts;
    // Component probes: Fibonacci points, golden angle pi (3 - sqrt 5),
    // joined when their dot product exceeds cos(2.5 sqrt(4 pi / N))
    // (arrangement.rs:327-391).
    const int np_ = ogk::kSasaProbes;
    std::vector<double> hp(3 * np_);
    const double golden = M_PI * (3.0 - std::sqrt(5.0));
    for (int k = 0; k < np_; ++k) {
      const double zz = 1.0 - (2.0 * k + 1.0) / np_;
      const double rr = std::sqrt(std::max(1.0 - zz * zz, 0.0));
      const double th = golden * k;
      hp[3 * k] = rr * std::cos(th);
      hp[3 * k + 1] = rr * std::sin(th);
      hp[3 * k + 2] = zz;
    }
    const double cos_thresh = std::cos(std::min(2.5 * std::sqrt(4.0 * M_PI / np_), M_PI));
    std::vector<int32_t> hpb(1, 0);
    std::vector<int16_t> hadj;
    for (int a = 0; a < np_; ++a) {
      for (int b = 0; b < np_; ++b) {
        if (a == b) continue;
        const double d = hp[3 * a] * hp[3 * b] + hp[3 * a + 1] * hp[3 * b + 1] + hp[3 * a + 2] * hp[3 * b + 2];
        if (d > cos_thresh) hadj.push_back(static_cast<int16_t>(b));
      }
      hpb.push_back(static_cast<int32_t>(hadj.size()));
    }
    OG_CUDA(e->sasa_probes.upload(hp, st));
    OG_CUDA(e->probe_begin.upload(hpb, st));
    OG_CUDA(e->probe_adj.upload(hadj, st));
    // Shrake-Rupley test points, the reference's 960 (sasa.rs:26).
    e->n_sr_dots = 960;
    OG_CUDA(e->sr_dots.upload(sr_dot_table(e->n_sr_dots), st));
    OG_CUDA(ogk::sasa_prepare());
  }

  // ---- learned Born radii: buffers when born_mode = 1 (the descriptor
  // class comes with the per-atom arrays)
  {
    OG_CUDA(ogk::tc_gemm_prepare());
    OG_CUDA(ogk::lgb_mlp_prepare());
    int dev = 0;
    OG_CUDA(cudaGetDevice(&dev));
    OG_CUDA(cudaDeviceGetAttribute(&e->n_sm, cudaDevAttrMultiProcessorCount, dev));
    const char* unf = std::getenv("OG_LGB_UNFUSED");
    e->lgb_unfused = unf && unf[0] == '1';
    if (e->p.born_mode == 1) {
      og_status ls = size_lgb_scratch(e, st);
      if (ls != OG_OK) return ls;
      OG_CUDA(e->lgb_params.alloc(ogk::kLgbNParams));
      OG_CUDA(e->lgb_part.alloc(2 * static_cast<size_t>(n_sys)));
    }
  }

  {
    og_status es = size_energy_scratch(e, st);
    if (es != OG_OK) return es;
  }

  // ---- per-system state
  std::vector<ogk::SysState> hs(n_sys);
  for (int si = 0; si < n_sys; ++si) hs[si] = sys_state_of(e, si);
  OG_CUDA(e->sys_state.upload(hs, st));

  // ---- pair work lists (build_pair_lists) and the persistent-launch queues
  OG_CUDA(e->pair_queue.alloc(2));
  {
    og_status ls = build_pair_lists(e, st);
    if (ls != OG_OK) return ls;
  }

  // ---- exclusion masks (per ordered tile pair) and the FP64 CSR
  {
    e->tile_refs.assign(e->n_tiles, {});
    e->excl_rows.assign(np, {});
    int t_min = 0, a_min = 0;
    std::set<int> touched;
    for (const auto& s : e->sys) mask_diagonal(e, s.tile_begin, s.tile_begin + s.n_tiles, &t_min, &touched);
    for (int si = 0; si < n_sys; ++si)
      for (size_t k = 0; k < e->sys[si].topo.excl_kind.size(); ++k) mask_exclusion(e, si, k, &t_min, &a_min, &touched);
    og_status xs = upload_exclusions(e, 0, 0, 0, 0, touched, st);
    if (xs != OG_OK) return xs;
  }

  // ---- bonded terms, reduction segments, SHAKE clusters
  for (int si = 0; si < n_sys; ++si) {
    og_status bs = append_bonded(e, si, TermSel::all(e->sys[si].topo), st);
    if (bs != OG_OK) return bs;
  }
  {
    og_status ss = upload_segments(e, st);
    if (ss != OG_OK) return ss;
  }
  OG_CUDA(e->seg_out.alloc(9 * static_cast<size_t>(n_sys)));  // energy terms: 5 per-atom + 4 bonded
  OG_CUDA(append(e->cl_start, std::vector<int32_t>(1, 0), st));
  if (e->p.constrain_h_bonds)
    for (int si = 0; si < n_sys; ++si) {
      og_status cs = append_clusters(e, si, TermSel::all(e->sys[si].topo).cons, {}, st);
      if (cs != OG_OK) return cs;
    }

  OG_CUDA(e->clamp_count.alloc(n_sys));
  OG_CUDA(e->sys_nonfinite.alloc(n_sys));
  OG_CUDA(cudaMemsetAsync(e->sys_nonfinite.p, 0, sizeof(int32_t) * n_sys, st));
  OG_CUDA(e->error_flag.alloc(1));
  OG_CUDA(cudaMemsetAsync(e->error_flag.p, 0, sizeof(int32_t), st));

  ogk::launch_pack(e->atoms(), true, st);
  og_status s2 = launch_check("pack");
  if (s2 != OG_OK) return s2;
  OG_CUDA(cudaStreamSynchronize(st));
  e->finalized = true;
  e->forces_valid = false;
  return OG_OK;
}

og_status eval_forces(og_engine* e) {
  if (e->p.born_mode == 1 && !e->lgb_params_set)
    return og_fail(OG_E_STATE, "born_mode 1 needs the network's parameters (og_lgb_set_params)");
  ogk::launch_pack(e->atoms(), true, e->stream);
  e->enqueue_forces();
  og_status st = launch_check("force evaluation");
  if (st != OG_OK) return st;
  e->forces_valid = true;
  return OG_OK;
}

void reset_graph(og_engine* e) {
  if (e->graph_exec) cudaGraphExecDestroy(e->graph_exec);
  if (e->graph) cudaGraphDestroy(e->graph);
  e->graph_exec = nullptr;
  e->graph = nullptr;
}

og_status lgb_check(og_engine* e) {
  if (e->p.born_mode == 1 && !e->lgb_params_set)
    return og_fail(OG_E_STATE, "born_mode 1 needs the network's parameters (og_lgb_set_params)");
  return OG_OK;
}

// Judge (plain GB against the network at the current positions): forces
// with plain radii are kept aside, forces with learned radii are evaluated
// last (they are the ones the next step uses), and the largest per-system
// RMS relative difference decides; above the tolerance the engine falls
// back to plain GB for good.
og_status lgb_judge(og_engine* e, double* err_out) {
  cudaStream_t st = e->stream;
  const int n_sys = static_cast<int>(e->sys.size());
  e->lgb_active = false;
  og_status s = eval_forces(e);
  if (s != OG_OK) return s;
  const size_t bytes = sizeof(unsigned long long) * e->n_padded;
  OG_CUDA(cudaMemcpyAsync(e->lgb_fx.p, e->fx.p, bytes, cudaMemcpyDeviceToDevice, st));
  OG_CUDA(cudaMemcpyAsync(e->lgb_fy.p, e->fy.p, bytes, cudaMemcpyDeviceToDevice, st));
  OG_CUDA(cudaMemcpyAsync(e->lgb_fz.p, e->fz.p, bytes, cudaMemcpyDeviceToDevice, st));
  e->lgb_active = true;
  if ((s = eval_forces(e)) != OG_OK) return s;
  ogk::launch_lgb_force_error(e->fx.p, e->fy.p, e->fz.p, e->lgb_fx.p, e->lgb_fy.p, e->lgb_fz.p, e->seg_begin.p,
                              e->seg_end.p, n_sys, e->lgb_part.p, st);
  std::vector<double> part(2 * static_cast<size_t>(n_sys));
  OG_CUDA(cudaMemcpyAsync(part.data(), e->lgb_part.p, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, st));
  OG_CUDA(cudaStreamSynchronize(st));
  if ((s = launch_check("judge")) != OG_OK) return s;
  double err = 0.0;
  for (int k = 0; k < n_sys; ++k) err = std::max(err, std::sqrt(part[2 * k] / std::max(part[2 * k + 1], 1e-300)));
  e->lgb_last_err = err;
  e->lgb_judged += 1;
  e->lgb_since_judge = 0;
  if (!(err <= e->lgb_tol)) {
    e->lgb_active = false;
    reset_graph(e);
    if ((s = eval_forces(e)) != OG_OK) return s;
  }
  if (err_out) *err_out = err;
  return OG_OK;
}

og_status build_graph(og_engine* e) {
  if (e->graph_exec) return OG_OK;
  cudaStream_t cap;
  OG_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
  cudaStream_t saved = e->stream;
  e->stream = cap;
  cudaError_t err = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
  if (err == cudaSuccess) {
    e->enqueue_step();
    err = cudaStreamEndCapture(cap, &e->graph);
  }
  e->stream = saved;
  cudaStreamDestroy(cap);
  if (err != cudaSuccess) return cuda_fail(err, "graph capture");
  // Kernel nodes run at the launch stream's priority: the surface term's
  // blocks, launched first, are dispatched first and the pair kernels fill
  // its tail.  (Honouring the captured node priorities, pair kernels first,
  // measured slower: they displace surface warps, whose latency-bound work
  // then stretches the step.)
  OG_CUDA(cudaGraphInstantiate(&e->graph_exec, e->graph, 0));
  return OG_OK;
}

// ---- co-translational growth

// Whether `grown` extends `base`: more atoms, the first base.n with the same
// parameters bit for bit, and, in every term list (bonds, angles, dihedrals
// with their Fourier terms, impropers, exclusions, constraints), the records
// among those atoms equal to base's records in base's order (a grown chain's
// topology lists them so: appending a residue adds atoms after the old ones
// and terms that touch them).  On success `d` lists the records of `grown`
// that touch a new atom, in grown's order; else the reason is returned.
std::string topology_delta(const TopoCopy& base, const TopoCopy& grown, TermSel* d) {
  const int n_old = base.n;
  if (grown.n <= n_old) return "the grown topology has no new atoms";
  auto same_prefix = [n_old](const auto& a, const auto& b) {
    return std::memcmp(a.data(), b.data(), sizeof(a[0]) * static_cast<size_t>(n_old)) == 0;
  };
  if (!same_prefix(base.charge, grown.charge) || !same_prefix(base.rmin, grown.rmin) ||
      !same_prefix(base.eps, grown.eps) || !same_prefix(base.rmin14, grown.rmin14) ||
      !same_prefix(base.eps14, grown.eps14) || !same_prefix(base.rho, grown.rho) ||
      !same_prefix(base.scale, grown.scale) || !same_prefix(base.mass, grown.mass) ||
      !same_prefix(base.element, grown.element))
    return "the parameters of the existing atoms differ";
  // One list: `arity` atom indices per record; same(g, b) compares the
  // records' parameters.
  auto split = [n_old](const char* what, int arity, const std::vector<int32_t>& ga, const std::vector<int32_t>& ba,
                       auto same, std::vector<int>* out) -> std::string {
    const size_t gn = ga.size() / arity, bn = ba.size() / arity;
    size_t k = 0;
    for (size_t g = 0; g < gn; ++g) {
      bool is_new = false;
      for (int c = 0; c < arity; ++c) is_new |= ga[g * arity + c] >= n_old;
      if (is_new) {
        out->push_back(static_cast<int>(g));
        continue;
      }
      bool eq = k < bn && same(g, k);
      for (int c = 0; eq && c < arity; ++c) eq = ga[g * arity + c] == ba[k * arity + c];
      if (!eq) return std::string(what) + " among the existing atoms differ";
      ++k;
    }
    if (k != bn) return std::string(what) + " among the existing atoms differ";
    return "";
  };
  std::string why;
  why = split("bonds", 2, grown.bonds, base.bonds, [&](size_t g, size_t b) {
    return grown.bond_k[g] == base.bond_k[b] && grown.bond_r0[g] == base.bond_r0[b];
  }, &d->bonds);
  if (!why.empty()) return why;
  why = split("angles", 3, grown.angles, base.angles, [&](size_t g, size_t b) {
    return grown.angle_k[g] == base.angle_k[b] && grown.angle_t0[g] == base.angle_t0[b];
  }, &d->angles);
  if (!why.empty()) return why;
  why = split("dihedrals", 4, grown.dihedrals, base.dihedrals, [&](size_t g, size_t b) {
    const int g0 = grown.dih_start[g], g1 = grown.dih_start[g + 1], b0 = base.dih_start[b], b1 = base.dih_start[b + 1];
    if (g1 - g0 != b1 - b0) return false;
    for (int m = 0; m < g1 - g0; ++m)
      if (grown.term_k[g0 + m] != base.term_k[b0 + m] || grown.term_n[g0 + m] != base.term_n[b0 + m] ||
          grown.term_delta[g0 + m] != base.term_delta[b0 + m])
        return false;
    return true;
  }, &d->dihedrals);
  if (!why.empty()) return why;
  why = split("impropers", 4, grown.impropers, base.impropers, [&](size_t g, size_t b) {
    return grown.imp_k[g] == base.imp_k[b] && grown.imp_psi0[g] == base.imp_psi0[b];
  }, &d->impropers);
  if (!why.empty()) return why;
  why = split("exclusions", 2, grown.excl, base.excl,
              [&](size_t g, size_t b) { return grown.excl_kind[g] == base.excl_kind[b]; }, &d->excl);
  if (!why.empty()) return why;
  return split("constraints", 2, grown.cons, base.cons,
               [&](size_t g, size_t b) { return grown.cons_d[g] == base.cons_d[b]; }, &d->cons);
}

// og_engine_append_atoms: system si (the engine's last) takes the atoms and
// terms that `grown` adds.  Only what the new atoms touch changes on the
// device: the per-atom tables from the tile holding the first new atom on,
// the new atoms' positions and velocities, the exclusion-mask blocks and
// CSR rows the new exclusions reach, the new bonded terms and SHAKE clusters
// appended to their lists, the system's reduction segments and state.  The
// existing atoms' positions, velocities and step count stay where they are
// on the device.  The pair work lists are rebuilt only when the system gains
// a tile.
og_status append_impl(og_engine* e, int si, const TopoCopy& grown, const double* xyz_new, const double* v_new) {
  SysHost& sh = e->sys[si];
  TermSel d;
  const std::string why = topology_delta(sh.topo, grown, &d);
  if (!why.empty()) return og_fail(OG_E_BADARG, "og_engine_append_atoms: " + why);
  cudaStream_t st = e->stream;
  const int n_old = sh.topo.n, n_new = grown.n, n_add = n_new - n_old;
  const int old_tiles = e->n_tiles, old_np = e->n_padded;
  std::set<int> old_heavy;  // system-local heavy atoms with a SHAKE cluster on the device
  for (size_t k = 0; k < sh.topo.cons_d.size(); ++k) {
    const int a = sh.topo.cons[2 * k], b = sh.topo.cons[2 * k + 1];
    old_heavy.insert(sh.topo.element[a] == 0 ? b : a);
  }
  sh.topo = grown;
  sh.xyz.resize(3 * static_cast<size_t>(n_old));
  sh.xyz.insert(sh.xyz.end(), xyz_new, xyz_new + 3 * static_cast<size_t>(n_add));
  sh.n_tiles = (n_new + kTile - 1) / kTile;
  const int np = sh.atom_begin + sh.n_tiles * kTile;
  e->n_padded = np;
  e->n_tiles = np / kTile;

  // per-atom arrays: grown in place (contents kept), then the static tables
  // of the tiles from the first new atom's on and the new atoms' state
  for (auto* v : {&e->x, &e->y, &e->z, &e->vx, &e->vy, &e->vz, &e->rx, &e->ry, &e->rz, &e->mass, &e->inv_mass,
                  &e->q, &e->rmin, &e->eps, &e->rmin14, &e->eps14, &e->rho, &e->rho_tilde, &e->srho, &e->born_r,
                  &e->born_r64, &e->integral64, &e->e_lj, &e->e_coul, &e->e_gb, &e->e_self, &e->sasa_r,
                  &e->sasa_gamma, &e->sasa_area, &e->sasa_energy})
    OG_CUDA(v->grow(np, st));
  for (auto* v : {&e->fx, &e->fy, &e->fz, &e->born_sum}) OG_CUDA(v->grow(np, st));
  for (auto* v : {&e->atom_sys, &e->local_idx, &e->atom_valid, &e->n_pairs, &e->lgb_class})
    OG_CUDA(v->grow(np, st));
  for (auto* v : {&e->pq, &e->lj, &e->gb}) OG_CUDA(v->grow(4 * static_cast<size_t>(np), st));
  OG_CUDA(e->origin.grow(e->n_tiles, st));
  const int a_first = sh.atom_begin + n_old;
  og_status s = fill_atoms(e, a_first / kTile * kTile, np, st);
  if (s == OG_OK) s = fill_positions(e, a_first, np, st);
  if (s != OG_OK) return s;
  if (v_new) {
    std::vector<double> hv[3];
    for (int c = 0; c < 3; ++c) {
      hv[c].resize(n_add);
      for (int k = 0; k < n_add; ++k) hv[c][k] = v_new[3 * k + c];
    }
    OG_CUDA(put(e->vx, a_first, hv[0], st));
    OG_CUDA(put(e->vy, a_first, hv[1], st));
    OG_CUDA(put(e->vz, a_first, hv[2], st));
  }
  {
    std::vector<int32_t> hmap(n_add);
    for (int k = 0; k < n_add; ++k) hmap[k] = a_first + k;
    OG_CUDA(append(e->real_map, hmap, st));
    e->n_real += n_add;
  }
  if (e->p.born_mode == 1 && (s = size_lgb_scratch(e, st)) != OG_OK) return s;
  if ((s = size_energy_scratch(e, st)) != OG_OK) return s;

  // surface term: task lists, scratch
  {
    std::vector<int32_t> htask, hall;
    sasa_lists(e, si, n_old, n_new, &htask, &hall);
    OG_CUDA(append(e->sasa_tasks, htask, st));
    OG_CUDA(append(e->sasa_all, hall, st));
    e->n_sasa_tasks += static_cast<int>(htask.size());
    e->n_sasa_all += static_cast<int>(hall.size());
    if ((s = size_sasa_scratch(e, st)) != OG_OK) return s;
    if ((s = upload_sys_tiles(e, st)) != OG_OK) return s;
  }

  // exclusions: the new tiles' diagonal blocks and the new exclusions
  {
    const int n_blocks = static_cast<int>(e->mask_of.size()), n_near = static_cast<int>(e->h_near.size());
    e->tile_refs.resize(e->n_tiles);
    e->excl_rows.resize(np);
    int t_min = e->n_tiles, a_min = np;
    std::set<int> touched;
    mask_diagonal(e, old_tiles, e->n_tiles, &t_min, &touched);
    for (int k : d.excl) mask_exclusion(e, si, static_cast<size_t>(k), &t_min, &a_min, &touched);
    if ((s = upload_exclusions(e, n_blocks, std::min(t_min, old_tiles), std::min(a_min, old_np), n_near, touched,
                               st)) != OG_OK)
      return s;
  }

  // bonded terms and SHAKE clusters of the new atoms, appended
  if ((s = append_bonded(e, si, d, st)) != OG_OK) return s;
  if ((s = upload_segments(e, st)) != OG_OK) return s;
  if (e->p.constrain_h_bonds && (s = append_clusters(e, si, d.cons, old_heavy, st)) != OG_OK) return s;

  // the system's atom count and degrees of freedom (its step count, status
  // and temperature stay)
  {
    std::vector<ogk::SysState> hs;
    if ((s = read_status(e, &hs)) != OG_OK) return s;
    const ogk::SysState fresh = sys_state_of(e, si);
    hs[si].n_atoms = fresh.n_atoms;
    hs[si].dof_corr = fresh.dof_corr;
    OG_CUDA(cudaMemcpyAsync(e->sys_state.p + si, &hs[si], sizeof(ogk::SysState), cudaMemcpyHostToDevice, st));
  }

  if (e->n_tiles != old_tiles && (s = build_pair_lists(e, st)) != OG_OK) return s;
  ogk::launch_pack(e->atoms(), true, st);
  if ((s = launch_check("pack")) != OG_OK) return s;
  OG_CUDA(cudaStreamSynchronize(st));
  reset_graph(e);
  e->remd_ready = false;
  e->forces_valid = false;
  return OG_OK;
}

}  // namespace

extern "C" {

void og_params_default(og_params* p) {
  if (!p) return;
  *p = og_params{};
  p->nb_cutoff = 10.0;
  p->born_cutoff = 20.0;
  p->gb_force_cutoff = 10.0;
  p->dt_fs = 1.0;
  p->friction_ps_inv = 1.0;
  p->constrain_h_bonds = 0;
  p->shake_max_iters = 64;
  p->shake_tol_sq = 1e-6;
  p->include_sasa = 0;
  p->sasa_gamma_scale = 1.0;
  p->born_mode = 0;
  p->seed = 0;
}

og_status og_engine_create(const og_params* params, og_engine** out) {
  if (!params || !out) return og_fail(OG_E_BADARG, "null argument");
  *out = nullptr;
  if (!(params->dt_fs > 0.0)) return og_fail(OG_E_BADARG, "dt_fs must be positive");
  if (params->born_mode != 0 && params->born_mode != 1) return og_fail(OG_E_BADARG, "born_mode must be 0 or 1");
  int n_dev = 0;
  if (cudaGetDeviceCount(&n_dev) != cudaSuccess || n_dev == 0)
    return og_fail(OG_E_CUDA, "no CUDA device available");
  auto e = new (std::nothrow) og_engine();
  if (!e) return og_fail(OG_E_NOMEM, "engine allocation failed");
  e->p = *params;
  cudaError_t err = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking);
  if (err != cudaSuccess) {
    delete e;
    return cuda_fail(err, "cudaStreamCreate");
  }
  e->own_stream = true;
  *out = e;
  return OG_OK;
}

og_status og_engine_add_system(og_engine* e, const og_topology* topo, const double* xyz, double temperature_k,
                               int32_t* index) {
  if (!e || !topo || !xyz) return og_fail(OG_E_BADARG, "null argument");
  if (e->finalized) return og_fail(OG_E_STATE, "engine already finalized");
  if (!(temperature_k >= 0.0)) return og_fail(OG_E_BADARG, "temperature must be >= 0");
  SysHost s;
  og_status st = copy_topology(topo, &s.topo);
  if (st != OG_OK) return st;
  s.xyz.assign(xyz, xyz + 3 * static_cast<size_t>(topo->n_atoms));
  for (double v : s.xyz)
    if (!std::isfinite(v)) return og_fail(OG_E_NONFINITE, "initial positions are not finite");
  s.temperature = temperature_k;
  e->sys.push_back(std::move(s));
  if (index) *index = static_cast<int32_t>(e->sys.size()) - 1;
  return OG_OK;
}

og_status og_engine_finalize(og_engine* e) {
  if (!e) return og_fail(OG_E_BADARG, "null engine");
  if (e->finalized) return og_fail(OG_E_STATE, "engine already finalized");
  return finalize_impl(e);
}

og_status og_topology_extends(const og_topology* base, const og_topology* grown, int32_t* extends) {
  if (!base || !grown || !extends) return og_fail(OG_E_BADARG, "null argument");
  TopoCopy b, g;
  og_status st = copy_topology(base, &b);
  if (st == OG_OK) st = copy_topology(grown, &g);
  if (st != OG_OK) return st;
  TermSel d;
  const std::string why = topology_delta(b, g, &d);
  *extends = why.empty() ? 1 : 0;
  if (!why.empty()) og_fail(OG_E_BADARG, why);  // the reason, for og_last_error
  return OG_OK;
}

og_status og_engine_append_atoms(og_engine* e, int32_t s, const og_topology* grown, const double* xyz_new,
                                 const double* v_new) {
  og_status st = check_ready(e);
  if (st != OG_OK) return st;
  if (s != static_cast<int32_t>(e->sys.size()) - 1)
    return og_fail(OG_E_BADARG, "og_engine_append_atoms: only the engine's last system can grow");
  if (!grown || !xyz_new) return og_fail(OG_E_BADARG, "null argument");
  TopoCopy g;
  if ((st = copy_topology(grown, &g)) != OG_OK) return st;
  for (int k = 3 * e->sys[s].topo.n; k < 3 * g.n; ++k)
    if (!std::isfinite(xyz_new[k - 3 * e->sys[s].topo.n])) return og_fail(OG_E_BADARG, "non-finite position");
  return append_impl(e, s, g, xyz_new, v_new);
}

og_status og_engine_n_systems(const og_engine* e, int32_t* n) {
  if (!e || !n) return og_fail(OG_E_BADARG, "null argument");
  *n = static_cast<int32_t>(e->sys.size());
  return OG_OK;
}

og_status og_engine_set_stream(og_engine* e, void* stream) {
  if (!e) return og_fail(OG_E_BADARG, "null engine");
  OG_CUDA(cudaStreamSynchronize(e->stream));
  if (e->own_stream && e->stream) cudaStreamDestroy(e->stream);
  if (stream) {
    e->stream = static_cast<cudaStream_t>(stream);
    e->own_stream = false;
  } else {
    OG_CUDA(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
    e->own_stream = true;
  }
  return OG_OK;
}

og_status og_engine_synchronize(og_engine* e) {
  if (!e) return og_fail(OG_E_BADARG, "null engine");
  OG_CUDA(cudaStreamSynchronize(e->stream));
  return OG_OK;
}

void og_engine_destroy(og_engine* e) {
  if (!e) return;
  if (e->stream) cudaStreamSynchronize(e->stream);
  delete e;
}

og_status og_set_positions(og_engine* e, int32_t s, const double* xyz) {
  og_status st = check_sys(e, s);
  if (st != OG_OK) return st;
  if (!xyz) return og_fail(OG_E_BADARG, "null positions");
  st = set_xyz(e, s, e->x, e->y, e->z, xyz);
  e->forces_valid = false;
  return st;
}

og_status og_get_positions(og_engine* e, int32_t s, double* xyz) {
  og_status st = check_sys(e, s);
  if (st != OG_OK) return st;
  if (!xyz) return og_fail(OG_E_BADARG, "null positions");
  return get_xyz(e, s, e->x, e->y, e->z, xyz);
}

og_status og_set_velocities(og_engine* e, int32_t s, const double* v) {
  og_status st = check_sys(e, s);
  if (st != OG_OK) return st;
  if (!v) return og_fail(OG_E_BADARG, "null velocities");
  return set_xyz(e, s, e->vx, e->vy, e->vz, v);
}

og_status og_get_velocities(og_engine* e, int32_t s, double* v) {
  og_status st = check_sys(e, s);
  if (st != OG_OK) return st;
  if (!v) return og_fail(OG_E_BADARG, "null velocities");
  return get_xyz(e, s, e->vx, e->vy, e->vz, v);
}

og_status og_init_velocities(og_engine* e, int32_t s, uint64_t seed, int32_t remove_com) {
  og_status st = check_sys(e, s);
  if (st != OG_OK) return st;
  const SysHost& sh = e->sys[s];
  const int n = sh.topo.n;
  const double kbt = ogk::kBoltzmann * sh.temperature;
  Xoshiro rng(seed);
  std::vector<double> v(3 * static_cast<size_t>(n));
  for (int i = 0; i < n; ++i) {
    const double sigma = std::sqrt(kbt * ogk::kAccel / sh.topo.mass[i]);
    v[3 * i] = sigma * rng.gaussian();
    v[3 * i + 1] = sigma * rng.gaussian();
    v[3 * i + 2] = sigma * rng.gaussian();
  }
  if (remove_com) {
    double tm = 0.0, px = 0.0, py = 0.0, pz = 0.0;
    for (int i = 0; i < n; ++i) {
      px += v[3 * i] * sh.topo.mass[i];
      py += v[3 * i + 1] * sh.topo.mass[i];
      pz += v[3 * i + 2] * sh.topo.mass[i];
      tm += sh.topo.mass[i];
    }
    if (tm > 0.0) {
      const double cx = px / tm, cy = py / tm, cz = pz / tm;
      for (int i = 0; i < n; ++i) {
        v[3 * i] -= cx;
        v[3 * i + 1] -= cy;
        v[3 * i + 2] -= cz;
      }
    }
  }
  return set_xyz(e, s, e->vx, e->vy, e->vz, v.data());
}

og_status og_set_temperature(og_engine* e, int32_t s, double t) {
  og_status st = check_sys(e, s);
  if (st != OG_OK) return st;
  if (!(t >= 0.0)) return og_fail(OG_E_BADARG, "temperature must be >= 0");
  e->sys[s].temperature = t;
  const double kbt = ogk::kBoltzmann * t;
  OG_CUDA(cudaMemcpyAsync(reinterpret_cast<char*>(e->sys_state.p + s) + offsetof(ogk::SysState, temperature), &t,
                          sizeof(double), cudaMemcpyHostToDevice, e->stream));
  OG_CUDA(cudaMemcpyAsync(reinterpret_cast<char*>(e->sys_state.p + s) + offsetof(ogk::SysState, kbt), &kbt,
                          sizeof(double), cudaMemcpyHostToDevice, e->stream));
  OG_CUDA(cudaStreamSynchronize(e->stream));
  return OG_OK;
}

og_status og_set_tunnel(og_engine* e, const double* origin, const double* direction, double radius_a,
                        double length_a, double k_confine) {
  if (!e) return og_fail(OG_E_BADARG, "null engine");
  if (!origin || !direction) {
    e->tunnel_on = false;
  } else {
    if (!(radius_a >= 0.0) || !(length_a >= 0.0) || !std::isfinite(k_confine))
      return og_fail(OG_E_BADARG, "tunnel radius and length must be >= 0 and k finite");
    e->tunnel = ogk::TunnelParams{origin[0],    origin[1],    origin[2], direction[0], direction[1],
                                  direction[2], radius_a, length_a, k_confine};
    e->tunnel_on = true;
  }
  e->forces_valid = false;
  if (e->finalized) reset_graph(e);
  return OG_OK;
}

og_status og_compute_forces(og_engine* e, int32_t s, double* f_out) {
  og_status st = check_ready(e);
  if (st != OG_OK) return st;
  if (f_out && (s < 0 || s >= static_cast<int32_t>(e->sys.size())))
    return og_fail(OG_E_BADARG, "system index out of range");
  if ((st = eval_forces(e)) != OG_OK) return st;
  if (e->p.include_sasa) {
    std::vector<ogk::SysState> hs;
    if ((st = read_status(e, &hs)) != OG_OK) return st;
  }
  if (f_out) {
    const int n = e->sys[s].topo.n;
    std::vector<unsigned long long> h[3];
    const DVec<unsigned long long>* src[3] = {&e->fx, &e->fy, &e->fz};
    for (int c = 0; c < 3; ++c) {
      h[c].resize(n);
      if ((st = copy_sys_range(e, *src[c], s, h[c].data())) != OG_OK) return st;
    }
    OG_CUDA(cudaStreamSynchronize(e->stream));
    for (int i = 0; i < n; ++i)
      for (int c = 0; c < 3; ++c)
        f_out[3 * i + c] = static_cast<double>(static_cast<long long>(h[c][i])) * ogk::kForceUnscale;
  } else {
    OG_CUDA(cudaStreamSynchronize(e->stream));
  }
  return OG_OK;
}

og_status og_get_born_radii(og_engine* e, int32_t s, double* radii) {
  og_status st = check_sys(e, s);
  if (st != OG_OK) return st;
  if (!radii) return og_fail(OG_E_BADARG, "null output");
  if (!e->forces_valid && (st = eval_forces(e)) != OG_OK) return st;
  if ((st = copy_sys_range(e, e->born_r, s, radii)) != OG_OK) return st;
  OG_CUDA(cudaStreamSynchronize(e->stream));
  return OG_OK;
}

og_status og_get_born_integrals(og_engine* e, int32_t s, double* out) {
  og_status st = check_sys(e, s);
  if (st != OG_OK) return st;
  if (!out) return og_fail(OG_E_BADARG, "null output");
  if (!e->forces_valid && (st = eval_forces(e)) != OG_OK) return st;
  const int n = e->sys[s].topo.n;
  std::vector<unsigned long long> h(n);
  if ((st = copy_sys_range(e, e->born_sum, s, h.data())) != OG_OK) return st;
  OG_CUDA(cudaStreamSynchronize(e->stream));
  for (int i = 0; i < n; ++i) out[i] = static_cast<double>(static_cast<long long>(h[i])) * ogk::kBornUnscale;
  return OG_OK;
}

og_status og_compute_energies(og_engine* e, int32_t s, og_energies* out) {
  og_status st = check_ready(e);
  if (st != OG_OK) return st;
  const int n_sys = static_cast<int>(e->sys.size());
  if (!out) return og_fail(OG_E_BADARG, "null output");
  if (s < -1 || s >= n_sys) return og_fail(OG_E_BADARG, "system index out of range");
  cudaStream_t stream = e->stream;
  ogk::EnergyArgs a{};
  a.x = e->x.p; a.y = e->y.p; a.z = e->z.p; a.q = e->q.p;
  a.rmin = e->rmin.p; a.eps = e->eps.p; a.rmin14 = e->rmin14.p; a.eps14 = e->eps14.p;
  a.rho_tilde = e->rho_tilde.p; a.srho = e->srho.p; a.born_r = e->born_r64.p;
  a.atom_sys = e->atom_sys.p;
  std::vector<int32_t> hb(n_sys), hc(n_sys);
  for (int k = 0; k < n_sys; ++k) {
    hb[k] = e->sys[k].atom_begin;
    hc[k] = e->sys[k].topo.n;
  }
  DVec<int32_t> dbeg, dcnt;
  OG_CUDA(dbeg.upload(hb, stream));
  OG_CUDA(dcnt.upload(hc, stream));
  a.sys_begin = dbeg.p;
  a.sys_count = dcnt.p;
  a.excl_row = e->excl_row.p; a.excl_col = e->excl_col.p; a.excl_kind = e->excl_kind.p;
  a.n_atoms_padded = e->n_padded;
  a.nb_c2 = no_cutoff(e->p.nb_cutoff) ? INFINITY : e->p.nb_cutoff * e->p.nb_cutoff;
  a.born_c2 = no_cutoff(e->p.born_cutoff) ? INFINITY : e->p.born_cutoff * e->p.born_cutoff;
  const double rc = e->p.nb_cutoff;
  a.kappa = no_cutoff(rc) ? 0.0 : 1.0 / (2.0 * rc * rc * rc);
  a.crf = no_cutoff(rc) ? 0.0 : 3.0 / (2.0 * rc);
  a.integral = e->integral64.p;
  a.e_lj = e->e_lj.p; a.e_coul = e->e_coul.p; a.e_gb = e->e_gb.p; a.e_self = e->e_self.p;
  a.n_pairs = e->n_pairs.p;
  a.n_chunks = e->e_chunks; a.part = e->epart.p; a.part_pairs = e->epart_pairs.p;

  OG_CUDA(cudaMemsetAsync(e->clamp_count.p, 0, sizeof(int32_t) * n_sys, stream));
  ogk::launch_born64(a, stream);
  ogk::launch_born_finalize(e->atoms(), e->integral64.p, e->born_r64.p, false, e->clamp_count.p, stream);
  ogk::launch_energy64(a, stream);
  ogk::launch_bonded_energies(e->bonded_args(), stream);
  if (e->p.include_sasa) {
    OG_CUDA(cudaMemsetAsync(e->sasa_area.p, 0, sizeof(double) * e->n_padded, stream));
    OG_CUDA(cudaMemsetAsync(e->sasa_energy.p, 0, sizeof(double) * e->n_padded, stream));
    ogk::launch_pack(e->atoms(), false, stream);
    ogk::launch_sasa_areas(e->sasa_args(false), stream);
  }
  if ((st = launch_check("energy kernels")) != OG_OK) return st;

  // Deterministic per-system sums, all on the device, then one copy back:
  // seg_out = [lj | coulomb | gb pair | gb self | sasa | bond | angle |
  // dihedral | improper], n_sys each.
  const double* per_atom[5] = {e->e_lj.p, e->e_coul.p, e->e_gb.p, e->e_self.p, e->sasa_energy.p};
  const int n_terms = e->p.include_sasa ? 5 : 4;
  for (int k = 0; k < n_terms; ++k)
    ogk::launch_segment_sum(per_atom[k], e->seg_begin.p, e->seg_end.p, n_sys, e->seg_out.p + k * n_sys, stream);
  ogk::launch_segment_sum(e->bonded_e.p, e->seg_begin.p + n_sys, e->seg_end.p + n_sys, 4 * n_sys,
                          e->seg_out.p + 5 * n_sys, stream);
  std::vector<double> all(9 * static_cast<size_t>(n_sys), 0.0);
  OG_CUDA(cudaMemcpyAsync(all.data(), e->seg_out.p, sizeof(double) * (n_terms == 5 ? 9 : 4) * n_sys,
                          cudaMemcpyDeviceToHost, stream));
  if (n_terms < 5)
    OG_CUDA(cudaMemcpyAsync(all.data() + 5 * n_sys, e->seg_out.p + 5 * n_sys, sizeof(double) * 4 * n_sys,
                            cudaMemcpyDeviceToHost, stream));
  std::vector<double> sums[5];
  for (int k = 0; k < 5; ++k) sums[k].assign(all.begin() + k * n_sys, all.begin() + (k + 1) * n_sys);
  std::vector<double> bonded(all.begin() + 5 * n_sys, all.end());
  // Pair counts (int) summed on the host.
  std::vector<int32_t> clamp(n_sys);
  OG_CUDA(cudaMemcpyAsync(clamp.data(), e->clamp_count.p, sizeof(int32_t) * n_sys, cudaMemcpyDeviceToHost, stream));
  std::vector<int32_t> pairs(e->n_padded);
  OG_CUDA(cudaMemcpyAsync(pairs.data(), e->n_pairs.p, sizeof(int32_t) * e->n_padded, cudaMemcpyDeviceToHost,
                          stream));
  OG_CUDA(cudaStreamSynchronize(stream));
  if ((st = launch_check("energy reductions")) != OG_OK) return st;
  if (e->p.include_sasa) {
    std::vector<ogk::SysState> hs;
    if ((st = read_status(e, &hs)) != OG_OK) return st;
  }

  for (int k = 0; k < n_sys; ++k) {
    if (s >= 0 && k != s) continue;
    og_energies& o = out[s >= 0 ? 0 : k];
    o = og_energies{};
    o.bond = bonded[0 * n_sys + k];
    o.angle = bonded[1 * n_sys + k];
    o.dihedral = bonded[2 * n_sys + k];
    o.improper = bonded[3 * n_sys + k];
    o.lj = 0.5 * sums[0][k] * ogk::kKcalToKj;
    o.coulomb = 0.5 * sums[1][k] * ogk::kKcalToKj;
    o.gb_pair = 0.5 * sums[2][k] * ogk::kKcalToKj;
    o.gb_self = sums[3][k] * ogk::kKcalToKj;
    o.gb = o.gb_self + o.gb_pair;
    o.sasa = e->p.include_sasa ? sums[4][k] : 0.0;
    o.total = o.bond + o.angle + o.dihedral + o.improper + o.lj + o.coulomb + o.gb + o.sasa;
    o.born_clamped = clamp[k];
    long long np = 0;
    for (int i = e->sys[k].atom_begin; i < e->sys[k].atom_begin + e->sys[k].topo.n; ++i) np += pairs[i];
    o.nb_pairs = static_cast<int32_t>(np / 2);
  }
  return OG_OK;
}

og_status og_step(og_engine* e, int32_t n_steps) {
  og_status st = check_ready(e);
  if (st != OG_OK) return st;
  if (n_steps < 0) return og_fail(OG_E_BADARG, "negative step count");
  if ((st = lgb_check(e)) != OG_OK) return st;
  if (!e->forces_valid && (st = eval_forces(e)) != OG_OK) return st;
  int done = 0;
  while (done < n_steps) {
    // with learned radii, plain GB judges the forces every lgb_judge_interval steps
    int chunk = n_steps - done;
    const bool judging = e->lgb_on() && e->lgb_judge_interval > 0;
    if (judging) chunk = static_cast<int>(std::min<int64_t>(chunk, e->lgb_judge_interval - e->lgb_since_judge));
    if (e->profile) {
      for (int k = 0; k < chunk; ++k) e->enqueue_step();
      if ((st = launch_check("step")) != OG_OK) return st;
    } else if (chunk > 0) {
      if ((st = build_graph(e)) != OG_OK) return st;
      for (int k = 0; k < chunk; ++k) OG_CUDA(cudaGraphLaunch(e->graph_exec, e->stream));
    }
    done += chunk;
    if (judging) {
      e->lgb_since_judge += chunk;
      if (e->lgb_since_judge >= e->lgb_judge_interval) {
        double err = 0.0;
        if ((st = lgb_judge(e, &err)) != OG_OK) return st;
      }
    }
  }
  std::vector<ogk::SysState> hs;
  if ((st = read_status(e, &hs)) != OG_OK) return st;
  for (const auto& s : hs)
    if (s.status & ogk::kStatusDiverged) return og_fail(OG_E_NONFINITE, "a system diverged (non-finite velocity)");
  return OG_OK;
}

og_status og_system_stats(og_engine* e, int32_t s, int64_t* steps, int64_t* shake_failures, int32_t* diverged) {
  og_status st = check_sys(e, s);
  if (st != OG_OK) return st;
  std::vector<ogk::SysState> hs;
  if ((st = read_status(e, &hs)) != OG_OK) return st;
  if (steps) *steps = hs[s].steps;
  if (shake_failures) *shake_failures = hs[s].shake_failures;
  if (diverged) *diverged = (hs[s].status & ogk::kStatusDiverged) ? 1 : 0;
  return OG_OK;
}

og_status og_kinetic(og_engine* e, int32_t s, double* ke, double* temp) {
  og_status st = check_sys(e, s);
  if (st != OG_OK) return st;
  const int n_sys = static_cast<int>(e->sys.size());
  ogk::launch_kinetic(e->atoms(), e->seg_begin.p, e->seg_end.p, n_sys, e->seg_out.p, e->stream);
  std::vector<double> h(n_sys);
  OG_CUDA(cudaMemcpyAsync(h.data(), e->seg_out.p, sizeof(double) * n_sys, cudaMemcpyDeviceToHost, e->stream));
  OG_CUDA(cudaStreamSynchronize(e->stream));
  const double dof = 3.0 * e->sys[s].topo.n;
  if (ke) *ke = h[s];
  if (temp) *temp = dof > 0.0 ? 2.0 * h[s] / (dof * ogk::kBoltzmann) : 0.0;
  return OG_OK;
}

// ---------------------------------------------------------------- og_state
namespace {

og_status ensure_stage(og_engine* e) {
  const size_t n3 = 3 * static_cast<size_t>(e->n_real);
  if (e->stage_a.n != n3) OG_CUDA(e->stage_a.alloc(n3));
  if (e->stage_b.n != n3) OG_CUDA(e->stage_b.alloc(n3));
  if (e->stage_f.n != n3) OG_CUDA(e->stage_f.alloc(n3));
  return OG_OK;
}

}  // namespace

og_status og_engine_counts(const og_engine* e, int64_t* n_atoms, int32_t* n_systems) {
  og_status st = check_ready(e);
  if (st != OG_OK) return st;
  if (n_atoms) *n_atoms = e->n_real;
  if (n_systems) *n_systems = static_cast<int32_t>(e->sys.size());
  return OG_OK;
}

og_status og_get_state(og_engine* e, const og_state* out) {
  og_status st = check_ready(e);
  if (st != OG_OK) return st;
  if (!out) return og_fail(OG_E_BADARG, "null state");
  if ((st = ensure_stage(e)) != OG_OK) return st;
  const size_t bytes = sizeof(double) * 3 * static_cast<size_t>(e->n_real);
  cudaStream_t s = e->stream;
  if (out->positions) {
    ogk::launch_gather_xyz(e->x.p, e->y.p, e->z.p, e->real_map.p, e->n_real, e->stage_a.p, s);
    OG_CUDA(cudaMemcpyAsync(out->positions, e->stage_a.p, bytes, cudaMemcpyDeviceToHost, s));
  }
  if (out->velocities) {
    ogk::launch_gather_xyz(e->vx.p, e->vy.p, e->vz.p, e->real_map.p, e->n_real, e->stage_b.p, s);
    OG_CUDA(cudaMemcpyAsync(out->velocities, e->stage_b.p, bytes, cudaMemcpyDeviceToHost, s));
  }
  if (out->forces_fixed) {
    ogk::launch_gather_fixed(e->fx.p, e->fy.p, e->fz.p, e->real_map.p, e->n_real, e->stage_f.p, s);
    OG_CUDA(cudaMemcpyAsync(out->forces_fixed, e->stage_f.p, bytes, cudaMemcpyDeviceToHost, s));
  }
  if ((st = launch_check("state gather")) != OG_OK) return st;
  std::vector<ogk::SysState> hs;
  if ((st = read_status(e, &hs)) != OG_OK) return st;  // also waits for the copies
  for (size_t k = 0; k < hs.size(); ++k) {
    if (out->steps) out->steps[k] = hs[k].steps;
    if (out->shake_failures) out->shake_failures[k] = hs[k].shake_failures;
    if (out->status) out->status[k] = hs[k].status;
    if (out->temperature) out->temperature[k] = hs[k].temperature;
  }
  return OG_OK;
}

og_status og_set_state(og_engine* e, const og_state* in) {
  og_status st = check_ready(e);
  if (st != OG_OK) return st;
  if (!in) return og_fail(OG_E_BADARG, "null state");
  if ((st = ensure_stage(e)) != OG_OK) return st;
  const size_t bytes = sizeof(double) * 3 * static_cast<size_t>(e->n_real);
  cudaStream_t s = e->stream;
  if (in->positions) {
    OG_CUDA(cudaMemcpyAsync(e->stage_a.p, in->positions, bytes, cudaMemcpyHostToDevice, s));
    ogk::launch_scatter_xyz(e->stage_a.p, e->real_map.p, e->n_real, e->x.p, e->y.p, e->z.p, s);
  }
  if (in->velocities) {
    OG_CUDA(cudaMemcpyAsync(e->stage_b.p, in->velocities, bytes, cudaMemcpyHostToDevice, s));
    ogk::launch_scatter_xyz(e->stage_b.p, e->real_map.p, e->n_real, e->vx.p, e->vy.p, e->vz.p, s);
  }
  if (in->forces_fixed) {
    OG_CUDA(cudaMemcpyAsync(e->stage_f.p, in->forces_fixed, bytes, cudaMemcpyHostToDevice, s));
    ogk::launch_scatter_fixed(e->stage_f.p, e->real_map.p, e->n_real, e->fx.p, e->fy.p, e->fz.p, s);
  }
  if ((st = launch_check("state scatter")) != OG_OK) return st;
  if (in->steps || in->shake_failures || in->status || in->temperature) {
    std::vector<ogk::SysState> hs;
    if ((st = read_status(e, &hs)) != OG_OK) return st;
    for (size_t k = 0; k < hs.size(); ++k) {
      if (in->steps) hs[k].steps = in->steps[k];
      if (in->shake_failures) hs[k].shake_failures = in->shake_failures[k];
      if (in->status) hs[k].status = in->status[k];
      if (in->temperature) {
        if (!(in->temperature[k] >= 0.0)) return og_fail(OG_E_BADARG, "temperature must be >= 0");
        hs[k].temperature = in->temperature[k];
        hs[k].kbt = ogk::kBoltzmann * in->temperature[k];
        e->sys[k].temperature = in->temperature[k];
      }
    }
    OG_CUDA(cudaMemcpyAsync(e->sys_state.p, hs.data(), sizeof(ogk::SysState) * hs.size(), cudaMemcpyHostToDevice, s));
  }
  if (in->forces_fixed)
    e->forces_valid = true;
  else if (in->positions)
    e->forces_valid = false;
  OG_CUDA(cudaStreamSynchronize(s));  // the caller's buffers are free on return
  return OG_OK;
}

// ------------------------------------------------------------ checkpoints
namespace {

constexpr char kCkptMagic[8] = {'O', 'G', 'C', 'K', 'P', 'T', '0', '1'};
constexpr uint32_t kCkptVersion = 1;

struct HostState {
  std::vector<double> x, v, temp;
  std::vector<int64_t> f, steps, fails;
  std::vector<int32_t> status;
  explicit HostState(int64_t n, size_t n_sys)
      : x(3 * n), v(3 * n), temp(n_sys), f(3 * n), steps(n_sys), fails(n_sys), status(n_sys) {}
  og_state view() {
    return og_state{x.data(), v.data(), f.data(), steps.data(), fails.data(), status.data(), temp.data()};
  }
};

extern "C++" {
template <typename T>
bool put(FILE* f, const T* p, size_t n) { return std::fwrite(p, sizeof(T), n, f) == n; }
template <typename T>
bool get(FILE* f, T* p, size_t n) { return std::fread(p, sizeof(T), n, f) == n; }
}

}  // namespace

og_status og_save_checkpoint(og_engine* e, const char* path) {
  og_status st = check_ready(e);
  if (st != OG_OK) return st;
  if (!path) return og_fail(OG_E_BADARG, "null path");
  const size_t n_sys = e->sys.size();
  if (!e->forces_valid && (st = eval_forces(e)) != OG_OK) return st;
  HostState h(e->n_real, n_sys);
  const og_state v = h.view();
  if ((st = og_get_state(e, &v)) != OG_OK) return st;
  FILE* f = std::fopen(path, "wb");
  if (!f) return og_fail(OG_E_IO, std::string("cannot open ") + path);
  const int32_t ns = static_cast<int32_t>(n_sys);
  const int64_t na = e->n_real;
  std::vector<int32_t> counts;
  for (const auto& s : e->sys) counts.push_back(s.topo.n);
  const int32_t lgb_active = e->lgb_active ? 1 : 0;
  const int64_t since = e->lgb_since_judge;
  bool ok = put(f, kCkptMagic, 8) && put(f, &kCkptVersion, 1) && put(f, &ns, 1) && put(f, &na, 1) &&
            put(f, counts.data(), n_sys) && put(f, h.x.data(), h.x.size()) && put(f, h.v.data(), h.v.size()) &&
            put(f, h.f.data(), h.f.size()) && put(f, h.steps.data(), n_sys) && put(f, h.fails.data(), n_sys) &&
            put(f, h.status.data(), n_sys) && put(f, h.temp.data(), n_sys) && put(f, &lgb_active, 1) &&
            put(f, &since, 1);
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) return og_fail(OG_E_IO, std::string("checkpoint write failed: ") + path);
  return OG_OK;
}

og_status og_load_checkpoint(og_engine* e, const char* path) {
  og_status st = check_ready(e);
  if (st != OG_OK) return st;
  if (!path) return og_fail(OG_E_BADARG, "null path");
  FILE* f = std::fopen(path, "rb");
  if (!f) return og_fail(OG_E_IO, std::string("cannot open ") + path);
  const size_t n_sys = e->sys.size();
  char magic[8];
  uint32_t version = 0;
  int32_t ns = 0, lgb_active = 0;
  int64_t na = 0, since = 0;
  bool ok = get(f, magic, 8) && std::memcmp(magic, kCkptMagic, 8) == 0 && get(f, &version, 1) &&
            version == kCkptVersion && get(f, &ns, 1) && get(f, &na, 1);
  if (!ok) {
    std::fclose(f);
    return og_fail(OG_E_DATA, std::string("not an origami-b200 checkpoint: ") + path);
  }
  std::vector<int32_t> counts(ns > 0 ? ns : 0);
  ok = static_cast<size_t>(ns) == n_sys && na == e->n_real && get(f, counts.data(), counts.size());
  for (size_t k = 0; ok && k < n_sys; ++k) ok = counts[k] == e->sys[k].topo.n;
  if (!ok) {
    std::fclose(f);
    return og_fail(OG_E_BADARG, "checkpoint systems differ from the engine's");
  }
  HostState h(na, n_sys);
  ok = get(f, h.x.data(), h.x.size()) && get(f, h.v.data(), h.v.size()) && get(f, h.f.data(), h.f.size()) &&
       get(f, h.steps.data(), n_sys) && get(f, h.fails.data(), n_sys) && get(f, h.status.data(), n_sys) &&
       get(f, h.temp.data(), n_sys) && get(f, &lgb_active, 1) && get(f, &since, 1);
  std::fclose(f);
  if (!ok) return og_fail(OG_E_DATA, std::string("truncated checkpoint: ") + path);
  const og_state v = h.view();
  if ((st = og_set_state(e, &v)) != OG_OK) return st;
  if (!lgb_active && e->lgb_active) {
    e->lgb_active = false;  // the run had fallen back to plain GB
    reset_graph(e);
  }
  e->lgb_since_judge = since;
  return OG_OK;
}

// ---------------------------------------------------- trajectory capture
og_status og_trajectory_capture(og_trajectory* t, og_engine* e, int32_t s) {
  og_status st = check_sys(e, s);
  if (st != OG_OK) return st;
  if (!t) return og_fail(OG_E_BADARG, "null trajectory");
  const SysHost& sh = e->sys[s];
  if (sh.topo.n != t->layout.n_atoms) return og_fail(OG_E_BADARG, "system and chain atom counts differ");
  const size_t bytes = sizeof(double) * 3 * static_cast<size_t>(sh.topo.n);
  if (!t->staging) {
    OG_CUDA(cudaMalloc(reinterpret_cast<void**>(&t->staging), bytes));
    for (int k = 0; k < 2; ++k) {
      OG_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&t->pinned[k]), bytes, cudaHostAllocDefault));
      OG_CUDA(cudaEventCreateWithFlags(&t->copied[k], cudaEventDisableTiming));
    }
  }
  // the slot's previous frame (two captures ago) is written first; the
  // frame captured last stays in flight
  const int slot = static_cast<int>(t->captures & 1);
  if (t->pending[slot] >= 0 && (st = og_trajectory_flush(t, t->captures - 1)) != OG_OK) return st;
  int64_t first = 0;  // the system's first real atom
  for (int32_t k = 0; k < s; ++k) first += e->sys[k].topo.n;
  ogk::launch_gather_xyz(e->x.p, e->y.p, e->z.p, e->real_map.p + first, sh.topo.n, t->staging, e->stream);
  OG_CUDA(cudaMemcpyAsync(t->pinned[slot], t->staging, bytes, cudaMemcpyDeviceToHost, e->stream));
  OG_CUDA(cudaEventRecord(t->copied[slot], e->stream));
  if ((st = launch_check("trajectory gather")) != OG_OK) return st;
  t->pending[slot] = t->captures++;
  return OG_OK;
}

og_status og_remd_swap(og_engine* e, int32_t parity, const double* uniforms, int32_t* accepted) {
  og_status st = check_ready(e);
  if (st != OG_OK) return st;
  if (!uniforms) return og_fail(OG_E_BADARG, "null uniforms");
  const int n_sys = static_cast<int>(e->sys.size());
  std::vector<int> order(n_sys);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return e->sys[a].temperature < e->sys[b].temperature; });
  std::vector<og_energies> en(n_sys);
  if ((st = og_compute_energies(e, -1, en.data())) != OG_OK) return st;
  if (e->p.include_sasa) {
    // remd.rs:529-537: the swap energy's surface term is the Shrake-Rupley
    // energy (960 points, unscaled tension on C and S), summed in atom order.
    if ((st = sasa_areas_all(e, 1, e->sr_dots.p, e->n_sr_dots)) != OG_OK) return st;
    std::vector<double> area(e->n_padded);
    OG_CUDA(cudaMemcpyAsync(area.data(), e->sasa_area.p, sizeof(double) * e->n_padded, cudaMemcpyDeviceToHost,
                            e->stream));
    OG_CUDA(cudaStreamSynchronize(e->stream));
    const double g = 0.005 * ogk::kKcalToKj;
    for (int k = 0; k < n_sys; ++k) {
      const SysHost& sh = e->sys[k];
      double esr = 0.0;
      for (int a = 0; a < sh.topo.n; ++a) {
        const int el = sh.topo.element[a];
        if (el == 1 || el == 5) esr += g * area[sh.atom_begin + a];
      }
      en[k].total += esr - en[k].sasa;
    }
  }
  std::vector<ogk::SysState> hs;
  if ((st = read_status(e, &hs)) != OG_OK) return st;
  const int n_pairs = n_sys - 1;
  if (accepted)
    for (int k = 0; k < n_pairs; ++k) accepted[k] = 0;
  for (int pi = (parity & 1); pi < n_pairs; pi += 2) {
    const int a = order[pi], b = order[pi + 1];
    if ((hs[a].status | hs[b].status) & ogk::kStatusDiverged) continue;
    if (e->sys[a].topo.n != e->sys[b].topo.n) return og_fail(OG_E_BADARG, "replica exchange between unequal systems");
    const double ta = e->sys[a].temperature, tb = e->sys[b].temperature;
    const double beta_a = 1.0 / (ogk::kBoltzmann * ta), beta_b = 1.0 / (ogk::kBoltzmann * tb);
    const double delta = (beta_a - beta_b) * (en[a].total - en[b].total);
    const double p_acc = delta >= 0.0 ? 1.0 : std::exp(delta);
    if (uniforms[pi] < p_acc) {
      ogk::launch_swap_systems(e->atoms(), e->sys[a].atom_begin, e->sys[b].atom_begin, e->sys[a].topo.n,
                               std::sqrt(ta / tb), std::sqrt(tb / ta), e->stream);
      if (accepted) accepted[pi] = 1;
    }
  }
  if ((st = launch_check("replica swap")) != OG_OK) return st;
  OG_CUDA(cudaStreamSynchronize(e->stream));
  return OG_OK;
}

namespace {

// The FP64 energy kernels of og_compute_energies without its host reductions
// (their per-atom and per-term outputs stay on the device).
void enqueue_energy_kernels(og_engine* e, cudaStream_t stream) {
  ogk::EnergyArgs a{};
  a.x = e->x.p; a.y = e->y.p; a.z = e->z.p; a.q = e->q.p;
  a.rmin = e->rmin.p; a.eps = e->eps.p; a.rmin14 = e->rmin14.p; a.eps14 = e->eps14.p;
  a.rho_tilde = e->rho_tilde.p; a.srho = e->srho.p; a.born_r = e->born_r64.p;
  a.atom_sys = e->atom_sys.p;
  a.sys_begin = e->remd_begin.p;
  a.sys_count = e->remd_count.p;
  a.excl_row = e->excl_row.p; a.excl_col = e->excl_col.p; a.excl_kind = e->excl_kind.p;
  a.n_atoms_padded = e->n_padded;
  a.nb_c2 = no_cutoff(e->p.nb_cutoff) ? INFINITY : e->p.nb_cutoff * e->p.nb_cutoff;
  a.born_c2 = no_cutoff(e->p.born_cutoff) ? INFINITY : e->p.born_cutoff * e->p.born_cutoff;
  const double rc = e->p.nb_cutoff;
  a.kappa = no_cutoff(rc) ? 0.0 : 1.0 / (2.0 * rc * rc * rc);
  a.crf = no_cutoff(rc) ? 0.0 : 3.0 / (2.0 * rc);
  a.integral = e->integral64.p;
  a.e_lj = e->e_lj.p; a.e_coul = e->e_coul.p; a.e_gb = e->e_gb.p; a.e_self = e->e_self.p;
  a.n_pairs = e->n_pairs.p;
  a.n_chunks = e->e_chunks; a.part = e->epart.p; a.part_pairs = e->epart_pairs.p;
  ogk::launch_born64(a, stream);
  ogk::launch_born_finalize(e->atoms(), e->integral64.p, e->born_r64.p, false, e->clamp_count.p, stream);
  ogk::launch_energy64(a, stream);
  ogk::launch_bonded_energies(e->bonded_args(), stream);
}

}  // namespace

og_status og_remd_run(og_engine* e, int32_t n_rounds, int32_t steps_per_swap, uint64_t seed, int64_t* attempts,
                      int64_t* accepts, int32_t* sys_of_slot) {
  og_status st = check_ready(e);
  if (st != OG_OK) return st;
  const int n = static_cast<int>(e->sys.size());
  if (n_rounds < 0 || steps_per_swap < 1) return og_fail(OG_E_BADARG, "og_remd_run: n_rounds >= 0, steps_per_swap >= 1");
  if (e->p.include_sasa)
    return og_fail(OG_E_UNSUPPORTED, "og_remd_run: the surface term's swap energy (Shrake-Rupley) is og_remd_swap's");
  for (const auto& sh : e->sys)
    if (sh.topo.n != e->sys[0].topo.n) return og_fail(OG_E_BADARG, "replica exchange between unequal systems");
  cudaStream_t stream = e->stream;
  if (!e->remd_ready) {
    std::vector<int32_t> order(n), hb(n), hc(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return e->sys[a].temperature < e->sys[b].temperature; });
    std::vector<double> temps(n);
    for (int k = 0; k < n; ++k) {
      temps[k] = e->sys[order[k]].temperature;
      hb[k] = e->sys[k].atom_begin;
      hc[k] = e->sys[k].topo.n;
    }
    OG_CUDA(e->remd_slot.upload(order, stream));
    OG_CUDA(e->remd_temps.upload(temps, stream));
    OG_CUDA(e->remd_begin.upload(hb, stream));
    OG_CUDA(e->remd_count.upload(hc, stream));
    OG_CUDA(e->remd_total.alloc(n));
    OG_CUDA(e->remd_vscale.alloc(n));
    OG_CUDA(e->remd_attempts.alloc(std::max(n - 1, 1)));
    OG_CUDA(e->remd_accepts.alloc(std::max(n - 1, 1)));
    OG_CUDA(cudaMemsetAsync(e->remd_attempts.p, 0, sizeof(long long) * std::max(n - 1, 1), stream));
    OG_CUDA(cudaMemsetAsync(e->remd_accepts.p, 0, sizeof(long long) * std::max(n - 1, 1), stream));
    e->remd_ready = true;
    e->remd_round = 0;
  }
  ogk::RemdArgs r{};
  r.sys = e->sys_state.p;
  r.sys_of_slot = e->remd_slot.p;
  r.temps = e->remd_temps.p;
  r.total = e->remd_total.p;
  r.vscale = e->remd_vscale.p;
  r.attempts = e->remd_attempts.p;
  r.accepts = e->remd_accepts.p;
  r.e_lj = e->e_lj.p; r.e_coul = e->e_coul.p; r.e_gb = e->e_gb.p; r.e_self = e->e_self.p;
  r.bonded_e = e->bonded_e.p;
  r.seg_begin = e->seg_begin.p;
  r.seg_end = e->seg_end.p;
  r.n_slots = n;
  r.seed = seed;
  for (int round = 0; round < n_rounds; ++round) {
    if ((st = og_step(e, steps_per_swap)) != OG_OK && st != OG_E_NONFINITE) return st;
    enqueue_energy_kernels(e, stream);
    ogk::launch_remd_round(e->atoms(), r, static_cast<int>(e->remd_round & 1u), e->remd_round, stream);
    e->remd_round += 1;
    if ((st = launch_check("replica exchange")) != OG_OK) return st;
  }
  std::vector<long long> ha(std::max(n - 1, 1)), hac(std::max(n - 1, 1));
  OG_CUDA(cudaMemcpyAsync(ha.data(), e->remd_attempts.p, sizeof(long long) * ha.size(), cudaMemcpyDeviceToHost,
                          stream));
  OG_CUDA(cudaMemcpyAsync(hac.data(), e->remd_accepts.p, sizeof(long long) * hac.size(), cudaMemcpyDeviceToHost,
                          stream));
  std::vector<int32_t> slots(n);
  OG_CUDA(cudaMemcpyAsync(slots.data(), e->remd_slot.p, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, stream));
  std::vector<ogk::SysState> hs;
  if ((st = read_status(e, &hs)) != OG_OK) return st;  // synchronises
  for (int k = 0; k < n; ++k) e->sys[k].temperature = hs[k].temperature;
  for (int k = 0; k + 1 < n; ++k) {
    if (attempts) attempts[k] = ha[k];
    if (accepts) accepts[k] = hac[k];
  }
  if (sys_of_slot)
    for (int k = 0; k < n; ++k) sys_of_slot[k] = slots[k];
  return OG_OK;
}

og_status og_compute_sasa(og_engine* e, int32_t s, int32_t method, int32_t n_dots, double* area_out) {
  og_status st = check_sys(e, s);
  if (st != OG_OK) return st;
  if (!area_out) return og_fail(OG_E_BADARG, "null output");
  if (method != 0 && method != 1) return og_fail(OG_E_BADARG, "method must be 0 (PowerSasa) or 1 (Shrake-Rupley)");
  DVec<double> dots;
  const double* dp = e->sr_dots.p;
  int nd = e->n_sr_dots;
  if (method == 1 && n_dots > 0 && n_dots != e->n_sr_dots) {
    if (n_dots < 2) return og_fail(OG_E_BADARG, "n_dots must be >= 2");
    OG_CUDA(dots.upload(sr_dot_table(n_dots), e->stream));
    dp = dots.p;
    nd = n_dots;
  }
  if ((st = sasa_areas_all(e, method, dp, nd)) != OG_OK) return st;
  if ((st = copy_sys_range(e, e->sasa_area, s, area_out)) != OG_OK) return st;
  OG_CUDA(cudaStreamSynchronize(e->stream));
  return OG_OK;
}

og_status og_lgb_set_params(og_engine* e, const float* params) {
  og_status st = check_ready(e);
  if (st != OG_OK) return st;
  if (!params) return og_fail(OG_E_BADARG, "null parameters");
  if (e->p.born_mode != 1) return og_fail(OG_E_STATE, "the engine was not created with born_mode = 1");
  for (int k = 0; k < ogk::kLgbNParams; ++k)
    if (!std::isfinite(params[k])) return og_fail(OG_E_NONFINITE, "non-finite network parameter");
  OG_CUDA(cudaMemcpyAsync(e->lgb_params.p, params, sizeof(float) * ogk::kLgbNParams, cudaMemcpyHostToDevice,
                          e->stream));
  OG_CUDA(cudaStreamSynchronize(e->stream));
  if (!e->lgb_active) reset_graph(e);
  e->lgb_params_set = true;
  e->lgb_active = true;
  e->lgb_since_judge = 0;
  e->forces_valid = false;
  return OG_OK;
}

og_status og_lgb_set_judge(og_engine* e, int32_t interval_steps, double tolerance) {
  if (!e) return og_fail(OG_E_BADARG, "null engine");
  if (interval_steps < 0 || !(tolerance > 0.0)) return og_fail(OG_E_BADARG, "bad judge settings");
  e->lgb_judge_interval = interval_steps;
  e->lgb_tol = tolerance;
  return OG_OK;
}

og_status og_lgb_status(og_engine* e, int32_t* active, int32_t* judged, double* last_error) {
  if (!e) return og_fail(OG_E_BADARG, "null engine");
  if (active) *active = e->lgb_on() ? 1 : 0;
  if (judged) *judged = e->lgb_judged;
  if (last_error) *last_error = e->lgb_last_err;
  return OG_OK;
}

og_status og_lgb_judge(og_engine* e, double* rms_rel) {
  og_status st = check_ready(e);
  if (st != OG_OK) return st;
  if (!e->lgb_on()) return og_fail(OG_E_STATE, "learned radii are not active");
  return lgb_judge(e, rms_rel);
}

og_status og_lgb_samples(og_engine* e, int32_t s, float* x_out, float* target_out) {
  og_status st = check_ready(e);
  if (st != OG_OK) return st;
  const int n_sys = static_cast<int>(e->sys.size());
  if (s < -1 || s >= n_sys) return og_fail(OG_E_BADARG, "system index out of range");
  if (!x_out || !target_out) return og_fail(OG_E_BADARG, "null output");
  const int np = e->n_padded;
  if (!e->lgb_x.p) OG_CUDA(e->lgb_x.alloc(static_cast<size_t>(np) * ogk::kLgbIn));
  if (!e->lgb_rcfa.p) OG_CUDA(e->lgb_rcfa.alloc(np));
  // plain GB radii of the FP64 energy path (born_r64, every system) at the
  // current positions
  std::vector<og_energies> en(n_sys);
  if ((st = og_compute_energies(e, -1, en.data())) != OG_OK) return st;
  ogk::launch_pack(e->atoms(), false, e->stream);
  ogk::launch_lgb_descriptors(e->lgb_desc_args(), e->stream);
  if ((st = launch_check("descriptors")) != OG_OK) return st;
  std::vector<double> rc(np), rp(np);
  OG_CUDA(cudaMemcpyAsync(rc.data(), e->lgb_rcfa.p, sizeof(double) * np, cudaMemcpyDeviceToHost, e->stream));
  OG_CUDA(cudaMemcpyAsync(rp.data(), e->born_r64.p, sizeof(double) * np, cudaMemcpyDeviceToHost, e->stream));
  size_t row = 0;
  for (int k = 0; k < n_sys; ++k) {
    if (s >= 0 && k != s) continue;
    const SysHost& sh = e->sys[k];
    OG_CUDA(cudaMemcpyAsync(x_out + row * ogk::kLgbIn, e->lgb_x.p + static_cast<size_t>(sh.atom_begin) * ogk::kLgbIn,
                            sizeof(float) * ogk::kLgbIn * sh.topo.n, cudaMemcpyDeviceToHost, e->stream));
    row += sh.topo.n;
  }
  OG_CUDA(cudaStreamSynchronize(e->stream));
  row = 0;
  for (int k = 0; k < n_sys; ++k) {
    if (s >= 0 && k != s) continue;
    const SysHost& sh = e->sys[k];
    for (int a = 0; a < sh.topo.n; ++a)
      target_out[row + a] = static_cast<float>(std::log(rp[sh.atom_begin + a] / rc[sh.atom_begin + a]));
    row += sh.topo.n;
  }
  return OG_OK;
}

// ------------------------------------------------------------ autotuner
// Launch variants of the two pair passes, timed on the engine's own systems:
// CTA shape (i-tiles per CTA and the occupancy target), one CTA per work item
// or a persistent grid on a work queue, and the j-tile chunk of a work item.
// The best of each pass is kept in a JSON cache keyed by the workload's
// bucket (mode, total tiles and largest system's tiles rounded up to a power
// of two), so an engine with a cached bucket is configured without timing.

namespace {

int pow2_bucket(int x) {
  int b = 1;
  while (b < x) b <<= 1;
  return b;
}

std::string tune_key(const og_engine* e) {
  int max_tiles = 0;
  for (const auto& s : e->sys) max_tiles = std::max(max_tiles, s.n_tiles);
  const bool all_pairs = no_cutoff(e->p.nb_cutoff) && no_cutoff(e->p.gb_force_cutoff) && no_cutoff(e->p.born_cutoff);
  return std::string(all_pairs ? "all_pairs" : "cutoff") + "|tiles<=" + std::to_string(pow2_bucket(e->n_tiles)) +
         "|system_tiles<=" + std::to_string(pow2_bucket(max_tiles));
}

struct TuneEntry {
  int b[3], f[3];
  double born_ms, force_ms;
};

std::map<std::string, TuneEntry> read_tune_cache(const char* path) {
  std::map<std::string, TuneEntry> out;
  if (!path || !*path) return out;
  FILE* fh = std::fopen(path, "r");
  if (!fh) return out;
  char line[512], key[256];
  while (std::fgets(line, sizeof(line), fh)) {
    TuneEntry t{};
    if (std::sscanf(line, " \"%255[^\"]\": {\"born\": [%d, %d, %d], \"force\": [%d, %d, %d], \"born_ms\": %lf, "
                          "\"force_ms\": %lf}",
                    key, &t.b[0], &t.b[1], &t.b[2], &t.f[0], &t.f[1], &t.f[2], &t.born_ms, &t.force_ms) == 9)
      out[key] = t;
  }
  std::fclose(fh);
  return out;
}

bool write_tune_cache(const char* path, const std::map<std::string, TuneEntry>& m) {
  if (!path || !*path) return true;
  const std::string tmp = std::string(path) + ".tmp";
  FILE* fh = std::fopen(tmp.c_str(), "w");
  if (!fh) return false;
  std::fprintf(fh, "{\n");
  size_t k = 0;
  for (const auto& kv : m) {
    const TuneEntry& t = kv.second;
    std::fprintf(fh, " \"%s\": {\"born\": [%d, %d, %d], \"force\": [%d, %d, %d], \"born_ms\": %.6f, \"force_ms\": %.6f}%s\n",
                 kv.first.c_str(), t.b[0], t.b[1], t.b[2], t.f[0], t.f[1], t.f[2], t.born_ms, t.force_ms,
                 ++k < m.size() ? "," : "");
  }
  std::fprintf(fh, "}\n");
  const bool ok = std::fclose(fh) == 0;
  return ok && std::rename(tmp.c_str(), path) == 0;
}

// Median-free best of `reps` timed launches (after one untimed) of one pass
// variant, with the culled lists rebuilt in each launch in cutoff mode.
og_status time_pass(og_engine* e, bool born, const ogk::PairLaunch& lc, int chunk, int reps, double* best_ms) {
  cudaStream_t st = e->stream;
  DVec<ogk::PairWork> work;
  DVec<int32_t> jl, jl_cut, seg;
  DVec<ogk::CutBlock> cut;
  int n_work = 0, n_cut = 0;
  og_status s = build_pass_list(e, born ? 0 : 1, ogk::pair_shape_tiles(lc.shape), chunk, &work, &n_work, &jl, &cut,
                                &n_cut, &jl_cut, &seg, st);
  if (s != OG_OK) return s;
  ogk::PairArgs a = e->pair_args();
  a.work = work.p;
  a.n_work = n_work;
  a.jlist = jl.p;
  a.queue = e->pair_queue.p + (born ? 0 : 1);
  const double cutoff = born ? e->p.born_cutoff : std::max(e->p.nb_cutoff, e->p.gb_force_cutoff);
  const bool culled = born ? !no_cutoff(e->p.born_cutoff) : (!no_cutoff(e->p.nb_cutoff) && !no_cutoff(e->p.gb_force_cutoff));
  if (culled) {
    a.jlist = jl_cut.p;
    a.seg_end = seg.p;
  }
  cudaEvent_t t0, t1;
  OG_CUDA(cudaEventCreate(&t0));
  OG_CUDA(cudaEventCreate(&t1));
  double best = 1e30;
  for (int r = 0; r <= reps; ++r) {
    cudaEventRecord(t0, st);
    if (culled) ogk::launch_cut_lists(cut.p, n_cut, jl.p, e->origin.p, cutoff, jl_cut.p, seg.p, st);
    if (born)
      ogk::launch_born_pass(a, lc, st);
    else
      ogk::launch_force_pass(a, lc, st);
    cudaEventRecord(t1, st);
    cudaError_t err = cudaEventSynchronize(t1);
    if (err != cudaSuccess) {
      cudaEventDestroy(t0);
      cudaEventDestroy(t1);
      return cuda_fail(err, "autotune");
    }
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, t0, t1);
    if (r > 0) best = std::min(best, static_cast<double>(ms));
  }
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  og_status ls = launch_check("autotune");
  if (ls != OG_OK) return ls;
  *best_ms = best;
  return OG_OK;
}

og_status apply_launch(og_engine* e, const TuneEntry& t) {
  e->born_launch.shape = t.b[0];
  e->born_launch.persistent = t.b[1] != 0;
  e->chunk_b = t.b[2];
  e->force_launch.shape = t.f[0];
  e->force_launch.persistent = t.f[1] != 0;
  e->chunk_f = t.f[2];
  OG_CUDA(cudaStreamSynchronize(e->stream));
  og_status s = build_pair_lists(e, e->stream);
  if (s != OG_OK) return s;
  reset_graph(e);
  e->forces_valid = false;
  OG_CUDA(cudaStreamSynchronize(e->stream));
  return OG_OK;
}

bool valid_launch(int pass, int shape, int persistent, int chunk) {
  return shape >= 0 && shape < (pass == 0 ? ogk::kBornShapes : ogk::kForceShapes) &&
         (persistent == 0 || persistent == 1) && chunk >= 1 && chunk <= 4096;
}

}  // namespace

og_status og_engine_set_pair_launch(og_engine* e, int32_t pass, int32_t shape, int32_t persistent, int32_t chunk) {
  og_status s = check_ready(e);
  if (s != OG_OK) return s;
  if ((pass != 0 && pass != 1) || !valid_launch(pass, shape, persistent, chunk))
    return og_fail(OG_E_BADARG,
                   "og_engine_set_pair_launch: pass 0/1, shape 0..2 (Born) or 0..6 (force), persistent 0/1, chunk >= 1");
  TuneEntry t{{e->born_launch.shape, e->born_launch.persistent ? 1 : 0, e->chunk_b},
              {e->force_launch.shape, e->force_launch.persistent ? 1 : 0, e->chunk_f}, 0.0, 0.0};
  int* dst = pass == 0 ? t.b : t.f;
  dst[0] = shape;
  dst[1] = persistent;
  dst[2] = chunk;
  return apply_launch(e, t);
}

og_status og_engine_autotune(og_engine* e, const char* cache_path, og_autotune_result* out) {
  og_status s = check_ready(e);
  if (s != OG_OK) return s;
  const std::string key = tune_key(e);
  std::map<std::string, TuneEntry> cache = read_tune_cache(cache_path);
  TuneEntry best{};
  bool from_cache = false;
  double b_def = -1.0, f_def = -1.0;
  auto it = cache.find(key);
  if (it != cache.end() && valid_launch(0, it->second.b[0], it->second.b[1], it->second.b[2]) &&
      valid_launch(1, it->second.f[0], it->second.f[1], it->second.f[2])) {
    best = it->second;
    from_cache = true;
  } else {
    // Born radii at the current positions, so the force pass runs on real
    // data (the timed launches only add into accumulators that the next
    // force evaluation zeroes)
    ogk::launch_pack(e->atoms(), true, e->stream);
    ogk::PairArgs pb = e->pair_args();
    if (!no_cutoff(e->p.born_cutoff)) {
      ogk::launch_cut_lists(e->cut_b.p, e->n_cut_b, e->jlist.p, e->origin.p, e->p.born_cutoff, e->jlist_cut_b.p,
                            e->seg_end_b.p, e->stream);
      pb.jlist = e->jlist_cut_b.p;
      pb.seg_end = e->seg_end_b.p;
    }
    ogk::launch_born_pass(pb, e->born_launch, e->stream);
    ogk::launch_born_finalize(e->atoms(), nullptr, e->born_r.p, true, nullptr, e->stream);
    OG_CUDA(cudaStreamSynchronize(e->stream));
    const int chunks[3] = {8, 16, 32};
    for (int pass = 0; pass < 2; ++pass) {
      double bt = 1e30;
      int bc[3] = {0, 0, 16};
      for (int shape = 0; shape < (pass == 0 ? ogk::kBornShapes : ogk::kForceShapes); ++shape)
        for (int pers = 0; pers <= 1; ++pers)
          for (int chunk : chunks) {
            double ms = 0.0;
            ogk::PairLaunch lc;
            lc.shape = shape;
            lc.persistent = pers != 0;
            s = time_pass(e, pass == 0, lc, chunk, 3, &ms);
            if (s != OG_OK) return s;
            if (shape == 0 && pers == 0 && chunk == 16) (pass == 0 ? b_def : f_def) = ms;
            if (ms < bt) {
              bt = ms;
              bc[0] = shape;
              bc[1] = pers;
              bc[2] = chunk;
            }
          }
      int* dst = pass == 0 ? best.b : best.f;
      std::memcpy(dst, bc, sizeof(bc));
      (pass == 0 ? best.born_ms : best.force_ms) = bt;
    }
    cache[key] = best;
    if (!write_tune_cache(cache_path, cache)) return og_fail(OG_E_IO, std::string("cannot write ") + cache_path);
  }
  OG_CUDA(cudaMemsetAsync(e->sys_nonfinite.p, 0, sizeof(int32_t) * e->sys.size(), e->stream));
  s = apply_launch(e, best);
  if (s != OG_OK) return s;
  if (out) {
    out->born_shape = best.b[0];
    out->born_persistent = best.b[1];
    out->born_chunk = best.b[2];
    out->force_shape = best.f[0];
    out->force_persistent = best.f[1];
    out->force_chunk = best.f[2];
    out->born_ms = best.born_ms;
    out->force_ms = best.force_ms;
    out->born_ms_default = b_def;
    out->force_ms_default = f_def;
    out->from_cache = from_cache ? 1 : 0;
  }
  return OG_OK;
}

og_status og_profile_enable(og_engine* e, int32_t on) {
  if (!e) return og_fail(OG_E_BADARG, "null engine");
  e->profile = on != 0;
  e->prof.clear();
  return OG_OK;
}

og_status og_profile_read(og_engine* e, og_kernel_time* out, int32_t cap, int32_t* n_out) {
  if (!e || !n_out) return og_fail(OG_E_BADARG, "null argument");
  e->prof_names.clear();
  for (const auto& kv : e->prof) e->prof_names.push_back(kv.first);
  int k = 0;
  for (const auto& name : e->prof_names) {
    if (k >= cap) break;
    if (out) {
      out[k].name = name.c_str();
      out[k].ms = e->prof[name].first;
      out[k].launches = e->prof[name].second;
    }
    ++k;
  }
  *n_out = k;
  return OG_OK;
}

}  // extern "C"
