// Analytical PowerSasa on the GPU (FP64).  One warp owns one atom i: it
// gathers the caps that neighbouring expanded spheres cut from i's unit
// sphere, builds the exposed boundary (arcs and vertices) in shared memory,
// and then either scatters the gradient of A_i into the fixed-point force
// accumulators or evaluates A_i by Gauss-Bonnet.
//
// Restated from crates/energy/src/powersasa/:
//   geometry.rs      intersect_circles (:70-102), contains_strict
//   arrangement.rs   build_caps (:69-97), find_boundary (:100-227), helpers
//                    (:229-318), count_accessible_components (:327-391)
//   area.rs          bounded_area (:44-134), face walk (:140-222)
//   analytical.rs    build_atom_cache (:101-214), directional_area_derivative
//                    (:315-421), add_sasa_forces_analytical (:583-649)
//   derivatives.rs   via sasa_geom.h (reverse mode)
//
// Reorganisations of the reference's loops, each exact up to rounding:
//  * A cap whose circle lies inside another cap (by a margin far above
//    rounding) is dropped before the boundary is built.  Every point it
//    contains is strictly inside the larger cap, so every midpoint and probe
//    test gives the same answer, and the transitions it adds to other
//    circles lie strictly inside the larger cap, where they only split
//    buried segments.  The exposed arcs and vertices are unchanged.
//  * Transitions on a circle are ordered by a pseudo-angle (monotone in the
//    reference's atan2 angle, one division instead of an atan2), and the
//    exposure test point of the segment from a to b -- a rotated by half the
//    counter-clockwise angle about the cap axis -- comes from half-angle
//    identities of that angle's cosine and sine, so atan2 runs only for
//    exposed arcs' central angles.
//  * The gradient of A_i is taken term by term in reverse mode (sasa_geom.h)
//    instead of one forward directional derivative per (atom, axis).
#include <cmath>

#include "common.cuh"
#include "sasa.cuh"
#include "sasa_geom.h"

namespace ogk {

namespace {

using ogsasa::D3;
using ogsasa::cross;
using ogsasa::dot;
using ogsasa::norm;
using ogsasa::norm2;

constexpr unsigned kFull = 0xffffffffu;
constexpr int kWarps = 4;
constexpr double kPi = 3.14159265358979323846;

__device__ __forceinline__ D3 normalize(D3 a) { return a / norm(a); }

struct Cap {
  D3 axis;
  double c;
};

__device__ __forceinline__ bool contains_strict(Cap c, D3 p) { return dot(p, c.axis) > c.c + 1e-12; }

enum { kTwo = 0, kTangent = 1, kDisjoint = 2, kCoincident = 3 };

// geometry.rs:70-102 (one reciprocal for the shared denominator and one
// reciprocal square root for the normal's length; same values to rounding).
__device__ int intersect(Cap c1, Cap c2, D3* p, D3* q) {
  const double sigma = dot(c1.axis, c2.axis);
  const double denom = 1.0 - sigma * sigma;
  if (fabs(denom) < 1e-12) return fabs(c1.c - sigma * c2.c) < 1e-9 ? kCoincident : kDisjoint;
  const double inv = 1.0 / denom;
  const double a = (c1.c - sigma * c2.c) * inv;
  const double b = (c2.c - sigma * c1.c) * inv;
  const double c_sq = 1.0 - a * a - b * b - 2.0 * a * b * sigma;
  if (c_sq < -1e-9) return kDisjoint;
  const D3 base = c1.axis * a + c2.axis * b;
  if (fabs(c_sq) <= 1e-9) {
    *p = base;
    return kTangent;
  }
  const D3 nc = cross(c1.axis, c2.axis);
  const D3 off = nc * (sqrt(c_sq) * rsqrt(norm2(nc)));
  *p = base + off;
  *q = base - off;
  return kTwo;
}

__device__ __forceinline__ D3 helper_axis(D3 axis) {
  const double ax = fabs(axis.x), ay = fabs(axis.y), az = fabs(axis.z);
  if (ax < ay && ax < az) return {1.0, 0.0, 0.0};
  if (ay < az) return {0.0, 1.0, 0.0};
  return {0.0, 0.0, 1.0};
}

__device__ D3 sample_circle_point(Cap c) {
  const D3 h = helper_axis(c.axis);
  const D3 perp = normalize(h - c.axis * dot(h, c.axis));
  return c.axis * c.c + perp * sqrt(fmax(1.0 - c.c * c.c, 0.0));
}

// Monotone stand-in for atan2(y, x) on (-pi, pi]: range (-2, 2].
__device__ __forceinline__ double pseudo_angle(double x, double y) {
  const double d = fabs(x) + fabs(y);
  if (d == 0.0) return 0.0;
  const double r = x / d;
  return y >= 0.0 ? 1.0 - r : r - 1.0;
}

// identify_root_sign (derivatives.rs:117).
__device__ int identify_root_sign(Cap c1, Cap c2, D3 ref) {
  ogsasa::VpState sp, sm;
  if (!ogsasa::vp_forward(c1.axis, c1.c, c2.axis, c2.c, 1, &sp) ||
      !ogsasa::vp_forward(c1.axis, c1.c, c2.axis, c2.c, -1, &sm))
    return 1;
  return norm2(sp.v - ref) <= norm2(sm.v - ref) ? 1 : -1;
}

// ------------------------------------------------------ per-warp storage
struct WarpSmem {
  // caps (indices in neighbour order, i.e. ascending atom index)
  double cx[kSasaMaxCaps], cy[kSasaMaxCaps], cz[kSasaMaxCaps], cc[kSasaMaxCaps];
  int32_t owner[kSasaMaxCaps];
  uint8_t live[kSasaMaxCaps];
  // transitions of the cap being processed: sort key, unit radial direction
  double ta[kSasaMaxTrans], tx[kSasaMaxTrans], ty[kSasaMaxTrans], tz[kSasaMaxTrans];
  uint8_t tother[kSasaMaxTrans];
  uint8_t torder[kSasaMaxTrans];
  // exposed arcs
  double a_theta[kSasaMaxArcs], a_sx[kSasaMaxArcs], a_sy[kSasaMaxArcs], a_sz[kSasaMaxArcs];
  uint8_t a_cap[kSasaMaxArcs], a_full[kSasaMaxArcs], a_vis[kSasaMaxArcs];
  int16_t a_own[kSasaMaxArcs], a_vs[kSasaMaxArcs], a_ve[kSasaMaxArcs];
  // vertices (one per arc that is not a full circle)
  double v_x[kSasaMaxArcs], v_y[kSasaMaxArcs], v_z[kSasaMaxArcs];
  uint8_t v_in[kSasaMaxArcs], v_out[kSasaMaxArcs];
  int8_t v_sign[kSasaMaxArcs];
};

__device__ __forceinline__ Cap cap_at(const WarpSmem& w, int k) { return {{w.cx[k], w.cy[k], w.cz[k]}, w.cc[k]}; }
__device__ __forceinline__ D3 pos(const SasaArgs& a, int j) { return {a.x[j], a.y[j], a.z[j]}; }
// Unit radial direction of transition s of the circle being processed.
__device__ __forceinline__ D3 tpoint(const WarpSmem& w, int s) { return {w.tx[s], w.ty[s], w.tz[s]}; }

__device__ __forceinline__ int warp_excl_scan(int v, int lane, int* total) {
  int s = v;
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(kFull, s, o);
    if (lane >= o) s += t;
  }
  *total = __shfl_sync(kFull, s, 31);
  return s - v;
}

enum Outcome { kExposed = 0, kBuried = 1, kBounded = 2, kInvalid = 3 };

// A point of circle k (cos alpha_k = ck.c, radius sk = sin alpha_k) from its
// unit radial direction u (perpendicular to the axis).
__device__ __forceinline__ D3 circle_point(Cap ck, double sk, D3 u) { return ck.axis * ck.c + u * sk; }

// Segment of circle k from the transition with radial direction ua
// counter-clockwise to the one with ub (find_boundary's consecutive pair,
// arrangement.rs:190-215).  Returns false for a segment the reference skips
// (ccw < 1e-9); else the exposure test point *mid (ua rotated by half the ccw
// angle, midpoint_on_circle) and the cosine / sine of the ccw angle.
// single = the circle's only transition (the whole circle, ccw = 2 pi).
__device__ bool segment_midpoint(D3 ua, D3 ub, Cap ck, double sk, bool single, D3* mid, double* cos_ccw,
                                 double* sin_ccw) {
  if (single) {
    *cos_ccw = 1.0;
    *sin_ccw = 0.0;
    *mid = ck.axis * ck.c - ua * sk;
    return true;
  }
  const double c = dot(ua, ub);
  const double s = dot(ck.axis, cross(ua, ub));
  *cos_ccw = c;
  *sin_ccw = s;
  if (c > 0.0 && s >= 0.0 && s < 2e-9 && atan2(s, c) < 1e-9) return false;
  // cos / sin of half the ccw angle h in (0, pi], from c = cos 2h, s = sin 2h
  double ch, sh;
  if (c >= 0.0) {
    const double r = sqrt((1.0 + c) * 0.5);
    ch = s >= 0.0 ? r : -r;
    sh = fabs(s) / (2.0 * r);
  } else {
    sh = sqrt((1.0 - c) * 0.5);
    ch = s / (2.0 * sh);
  }
  *mid = circle_point(ck, sk, ua * ch + cross(ck.axis, ua) * sh);
  return true;
}

// Builds caps and the exposed boundary of atom i in w.  Returns the outcome;
// for kBounded, *n_arcs / *n_verts are the boundary sizes (possibly zero).
__device__ int build_boundary(const SasaArgs& a, WarpSmem& w, int i, int lane, int* n_arcs_out, int* n_verts_out,
                              int* n_live_out) {
  const int sys = a.atom_sys[i];
  const D3 pi = pos(a, i);
  const double ri = a.radius[i];
  const int2 st = a.sys_tiles[sys];

  // ---- caps (build_caps), neighbours in ascending atom order
  int n_caps = 0;
  bool enclosed = false;
  for (int t0 = 0; t0 < st.y; t0 += 32) {
    const int t = t0 + lane;
    bool hit = false;
    if (t < st.y) {
      const double4 o = a.origin[st.x + t];
      const double dx = o.x - pi.x, dy = o.y - pi.y, dz = o.z - pi.z;
      const double lim = o.w + ri + a.r_max + 1e-6;
      hit = dx * dx + dy * dy + dz * dz <= lim * lim;
    }
    unsigned hits = __ballot_sync(kFull, hit);
    while (hits) {
      const int b = __ffs(hits) - 1;
      hits &= hits - 1;
      const int j = (st.x + t0 + b) * 32 + lane;
      bool is_cap = false;
      double ax = 0.0, ay = 0.0, az = 0.0, ca = 0.0;
      if (j != i && a.atom_sys[j] >= 0) {
        const double dx = a.x[j] - pi.x, dy = a.y[j] - pi.y, dz = a.z[j] - pi.z;
        const double rj = a.radius[j];
        const double d = sqrt(dx * dx + dy * dy + dz * dz);
        if (d <= ri + rj) {
          if (d + ri <= rj) {
            enclosed = true;
          } else if (!(d + rj <= ri || d >= ri + rj)) {
            ca = (d * d + ri * ri - rj * rj) / (2.0 * d * ri);
            if (ca >= -1.0 && ca <= 1.0) {
              is_cap = true;
              ax = dx / d;
              ay = dy / d;
              az = dz / d;
            }
          }
        }
      }
      const unsigned caps = __ballot_sync(kFull, is_cap);
      if (is_cap) {
        const int slot = n_caps + __popc(caps & ((1u << lane) - 1u));
        if (slot < kSasaMaxCaps) {
          w.cx[slot] = ax;
          w.cy[slot] = ay;
          w.cz[slot] = az;
          w.cc[slot] = ca;
          w.owner[slot] = j;
        }
      }
      n_caps += __popc(caps);
    }
  }
  if (__any_sync(kFull, enclosed)) return kBuried;
  if (n_caps > kSasaMaxCaps) return kInvalid;
  if (n_caps == 0) return kExposed;
  __syncwarp();

  // ---- drop caps whose circle lies inside another cap: alpha_k < alpha_m
  // and angle(axis_k, axis_m) < alpha_m - alpha_k, i.e. sigma - c_k c_m -
  // margin > s_k s_m, compared squared (both sides positive)
  int n_live = 0;
  for (int k0 = 0; k0 < n_caps; k0 += 32) {
    const int k = k0 + lane;
    bool live = k < n_caps;
    if (live) {
      const double ck = w.cc[k], sk2 = 1.0 - ck * ck;
      const D3 ak = {w.cx[k], w.cy[k], w.cz[k]};
      for (int m = 0; m < n_caps; ++m) {
        const double cm = w.cc[m];
        if (m == k || !(ck > cm)) continue;
        const double lhs = ak.x * w.cx[m] + ak.y * w.cy[m] + ak.z * w.cz[m] - cm * ck - 1e-6;
        if (lhs > 0.0 && lhs * lhs > sk2 * (1.0 - cm * cm)) {
          live = false;
          break;
        }
      }
    }
    const unsigned lv = __ballot_sync(kFull, live);
    if (live) w.live[n_live + __popc(lv & ((1u << lane) - 1u))] = static_cast<uint8_t>(k);
    n_live += __popc(lv);
  }
  __syncwarp();

  // ---- boundary arcs, cap by cap (find_boundary)
  int n_arcs = 0, n_verts = 0;
  bool bad = false;
  for (int li = 0; li < n_live && !bad; ++li) {
    const int k = w.live[li];
    const Cap ck = cap_at(w, k);
    const D3 h = helper_axis(ck.axis);
    const D3 fu = normalize(h - ck.axis * dot(h, ck.axis));
    const D3 fv = cross(ck.axis, fu);
    // Transitions are kept as unit radial directions u: every one lies on
    // circle k, p = axis cos(alpha_k) + u sin(alpha_k).
    const double sk = sqrt(fmax(1.0 - ck.c * ck.c, 0.0));
    const double inv_sk = sk > 0.0 ? 1.0 / sk : 0.0;
    int n_tr = 0;
    for (int m0 = 0; m0 < n_live; m0 += 32) {
      const int lm = m0 + lane;
      int cnt = 0, m = -1;
      D3 p{}, q{};
      if (lm < n_live) {
        m = w.live[lm];
        if (m != k) {
          const double cm = w.cc[m];
          const double sig = ck.axis.x * w.cx[m] + ck.axis.y * w.cy[m] + ck.axis.z * w.cz[m];
          // (1 - sigma^2) c_sq; far below the tangency threshold means no
          // transition whatever the rounding.
          const double nn = 1.0 - sig * sig - ck.c * ck.c - cm * cm + 2.0 * sig * ck.c * cm;
          if (nn >= -1e-6) {
            const int kind = intersect(ck, cap_at(w, m), &p, &q);
            cnt = kind == kTwo ? 2 : (kind == kTangent ? 1 : 0);
          }
        }
      }
      int total;
      const int off = warp_excl_scan(cnt, lane, &total);
      if (n_tr + total > kSasaMaxTrans) {
        bad = true;
        break;
      }
      if (cnt >= 1) {
        const int s = n_tr + off;
        const D3 u = (p - ck.axis * ck.c) * inv_sk;
        w.ta[s] = pseudo_angle(dot(u, fu), dot(u, fv));
        w.tx[s] = u.x;
        w.ty[s] = u.y;
        w.tz[s] = u.z;
        w.tother[s] = static_cast<uint8_t>(m);
      }
      if (cnt == 2) {
        const int s = n_tr + off + 1;
        const D3 u = (q - ck.axis * ck.c) * inv_sk;
        w.ta[s] = pseudo_angle(dot(u, fu), dot(u, fv));
        w.tx[s] = u.x;
        w.ty[s] = u.y;
        w.tz[s] = u.z;
        w.tother[s] = static_cast<uint8_t>(m);
      }
      n_tr += total;
    }
    if (bad) break;
    __syncwarp();
    // stable sort by angle (ties keep push order)
    bool nonfinite = false;
    for (int s = lane; s < n_tr; s += 32) {
      const double as = w.ta[s];
      if (!isfinite(as)) nonfinite = true;
      int rank = 0;
      for (int t = 0; t < n_tr; ++t) {
        const double at = w.ta[t];
        rank += (at < as) || (at == as && t < s);
      }
      if (rank < kSasaMaxTrans) w.torder[rank] = static_cast<uint8_t>(s);
    }
    if (__any_sync(kFull, nonfinite)) {
      bad = true;
      break;
    }
    __syncwarp();
    // consecutive de-duplication (|dp|^2 < 1e-12 against the last kept;
    // |dp| = sin(alpha_k) |du| on the circle)
    const double sk2 = sk * sk;
    bool dup = false;
    for (int r = 1 + lane; r < n_tr; r += 32)
      dup |= norm2(tpoint(w, w.torder[r]) - tpoint(w, w.torder[r - 1])) * sk2 < 1e-12;
    int n_kept = n_tr;
    if (__any_sync(kFull, dup)) {
      if (lane == 0) {
        int kept = 0;
        for (int r = 0; r < n_tr; ++r) {
          const int s = w.torder[r];
          if (kept == 0 || norm2(tpoint(w, s) - tpoint(w, w.torder[kept - 1])) * sk2 >= 1e-12)
            w.torder[kept++] = static_cast<uint8_t>(s);
        }
        n_kept = kept;
      }
      n_kept = __shfl_sync(kFull, n_kept, 0);
      __syncwarp();
    }

    if (n_kept == 0) {
      // no vertices: the whole circle is exposed unless a probe on it is buried
      const D3 probe = sample_circle_point(ck);
      bool buried = false;
      for (int lm = lane; lm < n_live; lm += 32) {
        const int m = w.live[lm];
        if (m != k && contains_strict(cap_at(w, m), probe)) buried = true;
      }
      if (!__any_sync(kFull, buried)) {
        if (n_arcs >= kSasaMaxArcs) {
          bad = true;
          break;
        }
        if (lane == 0) {
          w.a_cap[n_arcs] = static_cast<uint8_t>(k);
          w.a_full[n_arcs] = 1;
          w.a_theta[n_arcs] = -2.0 * kPi;
          w.a_sx[n_arcs] = probe.x;
          w.a_sy[n_arcs] = probe.y;
          w.a_sz[n_arcs] = probe.z;
          w.a_own[n_arcs] = -1;
        }
        ++n_arcs;
      }
      __syncwarp();
      continue;
    }
    for (int r0 = 0; r0 < n_kept; r0 += 32) {
      const int r = r0 + lane;
      bool exposed = false;
      double cos_ccw = 1.0, sin_ccw = 0.0;
      int sa = 0, sb = 0;
      if (r < n_kept) {
        sa = w.torder[r];
        sb = w.torder[(r + 1) % n_kept];
        D3 mid;
        if (segment_midpoint(tpoint(w, sa), tpoint(w, sb), ck, sk, n_kept == 1, &mid, &cos_ccw, &sin_ccw)) {
          // A buried segment usually lies in one of the two caps whose
          // circles bound it; testing those first ends most searches early
          // (the answer -- inside any other cap -- does not depend on order).
          exposed = !contains_strict(cap_at(w, w.tother[sa]), mid) && !contains_strict(cap_at(w, w.tother[sb]), mid);
          for (int lm = 0; lm < n_live && exposed; ++lm) {
            const int m = w.live[lm];
            if (m != k && contains_strict(cap_at(w, m), mid)) exposed = false;
          }
        }
      }
      const unsigned ex = __ballot_sync(kFull, exposed);
      const int cnt = __popc(ex);
      if (n_arcs + cnt > kSasaMaxArcs) {
        bad = true;
        break;
      }
      if (exposed) {
        double ccw = atan2(sin_ccw, cos_ccw);
        if (ccw <= 0.0) ccw += 2.0 * kPi;
        const int rank = __popc(ex & ((1u << lane) - 1u));
        const int e = n_arcs + rank, v = n_verts + rank;
        w.a_cap[e] = static_cast<uint8_t>(k);
        w.a_full[e] = 0;
        w.a_theta[e] = -ccw;
        const D3 pb = circle_point(ck, sk, tpoint(w, sb)), pa = circle_point(ck, sk, tpoint(w, sa));
        w.a_sx[e] = pb.x;
        w.a_sy[e] = pb.y;
        w.a_sz[e] = pb.z;
        w.a_own[e] = static_cast<int16_t>(v);
        w.v_x[v] = pa.x;
        w.v_y[v] = pa.y;
        w.v_z[v] = pa.z;
        w.v_in[v] = static_cast<uint8_t>(k);
        w.v_out[v] = w.tother[sa];
      }
      n_arcs += cnt;
      n_verts += cnt;
    }
    __syncwarp();
  }
  if (bad) return kInvalid;
  __syncwarp();
  *n_arcs_out = n_arcs;
  *n_verts_out = n_verts;
  *n_live_out = n_live;
  return kBounded;
}

// Vertex signs and arc->vertex links (build_atom_cache).
__device__ void link_boundary(WarpSmem& w, int n_arcs, int n_verts, int lane) {
  for (int v = lane; v < n_verts; v += 32)
    w.v_sign[v] = static_cast<int8_t>(
        identify_root_sign(cap_at(w, w.v_in[v]), cap_at(w, w.v_out[v]), {w.v_x[v], w.v_y[v], w.v_z[v]}));
  for (int e = lane; e < n_arcs; e += 32) {
    int vs = -1, ve = -1;
    if (!w.a_full[e]) {
      const D3 s = {w.a_sx[e], w.a_sy[e], w.a_sz[e]};
      const int own = w.a_own[e];
      const D3 t = {w.v_x[own], w.v_y[own], w.v_z[own]};
      for (int v = 0; v < n_verts && (vs < 0 || ve < 0); ++v) {
        const D3 p = {w.v_x[v], w.v_y[v], w.v_z[v]};
        if (vs < 0 && norm2(p - s) < 1e-10) vs = v;
        if (ve < 0 && norm2(p - t) < 1e-10) ve = v;
      }
    }
    w.a_vs[e] = static_cast<int16_t>(vs);
    w.a_ve[e] = static_cast<int16_t>(ve);
  }
  __syncwarp();
}

__device__ __forceinline__ void scatter(const SasaArgs& a, int x, D3 g, double scale) {
  if (g.x != 0.0) add_fixed(a.fx + x, g.x * scale, kForceScale);
  if (g.y != 0.0) add_fixed(a.fy + x, g.y * scale, kForceScale);
  if (g.z != 0.0) add_fixed(a.fz + x, g.z * scale, kForceScale);
}

// Force path, stage 1: the boundary of atom i as term records
// (build_atom_cache + arc_other_cap_and_sign, analytical.rs:101-214, 655-670).
__global__ void __launch_bounds__(kWarps * 32, 4) k_sasa_boundary(SasaArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  WarpSmem& w = reinterpret_cast<WarpSmem*>(smem_raw)[warp];
  const int task = blockIdx.x * kWarps + warp;
  if (task >= a.n_tasks) return;
  const int i = a.tasks[task];
  const int sys = a.atom_sys[i];
  if (a.sys[sys].status & kStatusDiverged) return;
  int n_arcs = 0, n_verts = 0, n_live = 0;
  const int outcome = build_boundary(a, w, i, lane, &n_arcs, &n_verts, &n_live);
  if (outcome == kInvalid) {
    if (lane == 0) atomicOr(&a.sys[sys].status, kStatusSasaOverflow);
    return;
  }
  if (outcome != kBounded || n_arcs == 0) return;
  link_boundary(w, n_arcs, n_verts, lane);
  int arc_base = 0, vert_base = 0;
  if (lane == 0) {
    arc_base = atomicAdd(&a.counts[0], n_arcs);
    vert_base = atomicAdd(&a.counts[1], n_verts);
  }
  arc_base = __shfl_sync(kFull, arc_base, 0);
  vert_base = __shfl_sync(kFull, vert_base, 0);
  if (arc_base + n_arcs > a.term_cap || vert_base + n_verts > a.term_cap) {
    if (lane == 0) atomicOr(&a.sys[sys].status, kStatusSasaOverflow);
    return;
  }
  for (int e = lane; e < n_arcs; e += 32) {
    SasaArcTerm t;
    const int kc = w.a_cap[e];
    const int vs = w.a_vs[e], ve = w.a_ve[e];
    t.i = i;
    t.k = w.owner[kc];
    t.theta = w.a_theta[e];
    t.vertexed = (!w.a_full[e] && vs >= 0 && ve >= 0) ? 1 : 0;
    t.l = t.m = -1;
    t.ss = t.se = 1;
    t.pad = 0;
    if (t.vertexed) {
      const bool s_in = w.v_in[vs] == kc, e_in = w.v_in[ve] == kc;
      t.l = w.owner[s_in ? w.v_out[vs] : w.v_in[vs]];
      t.ss = s_in ? w.v_sign[vs] : -w.v_sign[vs];
      t.m = w.owner[e_in ? w.v_out[ve] : w.v_in[ve]];
      t.se = e_in ? w.v_sign[ve] : -w.v_sign[ve];
    }
    a.arc_terms[arc_base + e] = t;
  }
  for (int v = lane; v < n_verts; v += 32)
    a.vertex_terms[vert_base + v] = SasaVertexTerm{i, w.owner[w.v_in[v]], w.owner[w.v_out[v]], w.v_sign[v]};
}

// Force path, stage 2: one term per thread, F_x += gamma_i R_i^2 dTerm/dr_x.
__global__ void __launch_bounds__(128) k_sasa_terms(SasaArgs a) {
  const int n_arc = min(a.counts[0], a.term_cap), n_vert = min(a.counts[1], a.term_cap);
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n_arc + n_vert; t += gridDim.x * blockDim.x) {
    D3 gi = {0.0, 0.0, 0.0}, g1 = gi, g2 = gi, g3 = gi;
    int i, x1, x2, x3 = -1;
    if (t < n_arc) {
      const SasaArcTerm r = a.arc_terms[t];
      i = r.i;
      x1 = r.k;
      const D3 pi = pos(a, i);
      const double ri = a.radius[i];
      x2 = r.vertexed ? r.l : -1;
      x3 = r.vertexed ? r.m : -1;
      const D3 pl = r.vertexed ? pos(a, r.l) : pi, pm = r.vertexed ? pos(a, r.m) : pi;
      const double rl = r.vertexed ? a.radius[r.l] : ri, rm = r.vertexed ? a.radius[r.m] : ri;
      ogsasa::arc_gradient(pi, pos(a, x1), pl, pm, ri, a.radius[x1], rl, rm, r.ss, r.se, r.theta, r.vertexed != 0,
                           &gi, &g1, &g2, &g3);
    } else {
      const SasaVertexTerm r = a.vertex_terms[t - n_arc];
      i = r.i;
      x1 = r.k;
      x2 = r.l;
      ogsasa::vertex_gradient(pos(a, i), pos(a, x1), pos(a, x2), a.radius[i], a.radius[x1], a.radius[x2], r.sign,
                              &gi, &g1, &g2);
    }
    const double ri = a.radius[i];
    const double scale = a.gamma[i] * ri * ri;
    scatter(a, i, gi, scale);
    scatter(a, x1, g1, scale);
    if (x2 >= 0) scatter(a, x2, g2, scale);
    if (x3 >= 0) scatter(a, x3, g3, scale);
  }
}

// Face walk with tangent disambiguation (area.rs:140-222): loop count and
// the exterior-angle sum of the continuation actually taken.
__device__ void walk_faces(WarpSmem& w, int n_arcs, int lane, int* loops_out, double* vsum_out) {
  for (int e = lane; e < n_arcs; e += 32) w.a_vis[e] = 0;
  __syncwarp();
  int loops = 0;
  double vsum = 0.0;
  const double two_pi = 2.0 * kPi;
  for (int start = 0; start < n_arcs; ++start) {
    if (w.a_vis[start]) continue;
    if (w.a_full[start]) {
      __syncwarp();
      if (lane == 0) w.a_vis[start] = 1;
      __syncwarp();
      ++loops;
      continue;
    }
    int current = start;
    for (int guard = 0; guard <= n_arcs; ++guard) {
      __syncwarp();
      if (lane == 0) w.a_vis[current] = 1;
      __syncwarp();
      const int own = w.a_own[current];
      const D3 end_pt = {w.v_x[own], w.v_y[own], w.v_z[own]};
      const D3 t_in = normalize(cross(end_pt, cap_at(w, w.a_cap[current]).axis));
      int first = 1 << 30, best = 1 << 30;
      double best_ang = INFINITY;
      for (int c = lane; c < n_arcs; c += 32) {
        if (w.a_full[c]) continue;
        const D3 s = {w.a_sx[c], w.a_sy[c], w.a_sz[c]};
        if (!(norm2(s - end_pt) < 1e-10)) continue;
        if (c < first) first = c;
        if (c == current) continue;
        const D3 t_out = normalize(cross(end_pt, cap_at(w, w.a_cap[c]).axis));
        const double d = fmin(fmax(dot(t_in, t_out), -1.0), 1.0);
        double ang = atan2(dot(end_pt, cross(t_in, t_out)), d);
        if (ang <= 1e-9) ang += two_pi;
        if (ang < best_ang || (ang == best_ang && c < best)) {
          best_ang = ang;
          best = c;
        }
      }
      for (int o = 16; o > 0; o >>= 1) {
        const int f2 = __shfl_xor_sync(kFull, first, o);
        const double a2 = __shfl_xor_sync(kFull, best_ang, o);
        const int b2 = __shfl_xor_sync(kFull, best, o);
        first = min(first, f2);
        if (a2 < best_ang || (a2 == best_ang && b2 < best)) {
          best_ang = a2;
          best = b2;
        }
      }
      if (first == (1 << 30)) break;
      const int nxt = best < (1 << 30) ? best : first;
      const D3 t_out = normalize(cross(end_pt, cap_at(w, w.a_cap[nxt]).axis));
      const double d = fmin(fmax(dot(t_in, t_out), -1.0), 1.0);
      vsum += atan2(dot(end_pt, cross(t_in, t_out)), d);
      if (nxt == start) break;
      current = nxt;
    }
    ++loops;
  }
  *loops_out = loops;
  *vsum_out = vsum;
}

// count_accessible_components (arrangement.rs:327-391): accessible probes,
// then connected components of the fixed probe graph restricted to them by
// minimum-label propagation (the component count does not depend on how
// the components are found).
__device__ int count_components(const SasaArgs& a, WarpSmem& w, int n_live, int lane) {
  volatile int16_t* lab = reinterpret_cast<int16_t*>(w.ta);
  uint8_t* acc = reinterpret_cast<uint8_t*>(w.tx);
  bool any = false;
  for (int p = lane; p < kSasaProbes; p += 32) {
    const D3 pr = {a.probes[3 * p], a.probes[3 * p + 1], a.probes[3 * p + 2]};
    bool in = false;
    for (int lm = 0; lm < n_live && !in; ++lm) in = contains_strict(cap_at(w, w.live[lm]), pr);
    acc[p] = in ? 0 : 1;
    lab[p] = static_cast<int16_t>(in ? -1 : p);
    any |= !in;
  }
  if (!__any_sync(kFull, any)) return 0;
  __syncwarp();
  for (int iter = 0; iter < kSasaProbes; ++iter) {
    bool changed = false;
    for (int p = lane; p < kSasaProbes; p += 32) {
      if (!acc[p]) continue;
      int l = lab[p];
      for (int k = a.probe_adj_begin[p]; k < a.probe_adj_begin[p + 1]; ++k) {
        const int q = a.probe_adj[k];
        if (acc[q]) l = min(l, static_cast<int>(lab[q]));
      }
      if (l < lab[p]) {
        lab[p] = static_cast<int16_t>(l);
        changed = true;
      }
    }
    __syncwarp();
    if (!__any_sync(kFull, changed)) break;
  }
  int roots = 0;
  for (int p = lane; p < kSasaProbes; p += 32) roots += (acc[p] && lab[p] == p) ? 1 : 0;
  for (int o = 16; o > 0; o >>= 1) roots += __shfl_xor_sync(kFull, roots, o);
  return roots;
}

__global__ void __launch_bounds__(kWarps * 32) k_sasa_areas(SasaArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  WarpSmem& w = reinterpret_cast<WarpSmem*>(smem_raw)[warp];
  const int task = blockIdx.x * kWarps + warp;
  if (task >= a.n_tasks) return;
  const int i = a.tasks[task];
  const int sys = a.atom_sys[i];
  const double ri = a.radius[i];
  const double four_pi_r2 = 4.0 * kPi * ri * ri;
  int n_arcs = 0, n_verts = 0, n_live = 0;
  const int outcome = build_boundary(a, w, i, lane, &n_arcs, &n_verts, &n_live);
  double area = 0.0;
  if (outcome == kInvalid) {
    if (lane == 0) atomicOr(&a.sys[sys].status, kStatusSasaOverflow);
    area = NAN;
  } else if (outcome == kExposed) {
    area = four_pi_r2;
  } else if (outcome == kBounded && n_arcs > 0) {
    int loops;
    double vsum;
    walk_faces(w, n_arcs, lane, &loops, &vsum);
    if (loops > 0) {
      double arc_sum = 0.0;
      for (int e = 0; e < n_arcs; ++e) arc_sum += w.cc[w.a_cap[e]] * w.a_theta[e];
      int c = 1;
      if (loops >= 2) c = max(min(count_components(a, w, n_live, lane), loops), 1);
      const int chi = 2 * c - loops;
      area = ri * ri * (2.0 * kPi * chi - arc_sum - vsum);
      area = fmin(fmax(area, 0.0), four_pi_r2);
    }
  }
  if (lane == 0) {
    a.area[i] = area;
    a.energy[i] = a.gamma[i] * area;
  }
}

// Shrake-Rupley: one warp per atom, neighbours staged in shared memory,
// lanes over test points.
struct SrSmem {
  double nx[kSasaMaxCaps], ny[kSasaMaxCaps], nz[kSasaMaxCaps], nr2[kSasaMaxCaps];
};

__global__ void __launch_bounds__(kWarps * 32) k_shrake_rupley(SasaArgs a, const double* dots, int n_dots) {
  __shared__ SrSmem sm[kWarps];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  SrSmem& w = sm[warp];
  const int task = blockIdx.x * kWarps + warp;
  if (task >= a.n_tasks) return;
  const int i = a.tasks[task];
  const int sys = a.atom_sys[i];
  const D3 pi = pos(a, i);
  const double ri = a.radius[i];
  const int2 st = a.sys_tiles[sys];
  int n_nb = 0;
  for (int t0 = 0; t0 < st.y; t0 += 32) {
    const int t = t0 + lane;
    bool hit = false;
    if (t < st.y) {
      const double4 o = a.origin[st.x + t];
      const double dx = o.x - pi.x, dy = o.y - pi.y, dz = o.z - pi.z;
      const double lim = o.w + ri + a.r_max + 1e-6;
      hit = dx * dx + dy * dy + dz * dz <= lim * lim;
    }
    unsigned hits = __ballot_sync(kFull, hit);
    while (hits) {
      const int b = __ffs(hits) - 1;
      hits &= hits - 1;
      const int j = (st.x + t0 + b) * 32 + lane;
      bool nb = false;
      if (j != i && a.atom_sys[j] >= 0) nb = norm(pos(a, j) - pi) <= ri + a.radius[j];
      const unsigned m = __ballot_sync(kFull, nb);
      if (nb) {
        const int slot = n_nb + __popc(m & ((1u << lane) - 1u));
        if (slot < kSasaMaxCaps) {
          w.nx[slot] = a.x[j];
          w.ny[slot] = a.y[j];
          w.nz[slot] = a.z[j];
          w.nr2[slot] = a.radius[j] * a.radius[j];
        }
      }
      n_nb += __popc(m);
    }
  }
  if (n_nb > kSasaMaxCaps) {
    if (lane == 0) {
      atomicOr(&a.sys[sys].status, kStatusSasaOverflow);
      a.area[i] = NAN;
      a.energy[i] = NAN;
    }
    return;
  }
  __syncwarp();
  int acc = 0;
  for (int k = lane; k < n_dots; k += 32) {
    const D3 t = pi + D3{dots[3 * k], dots[3 * k + 1], dots[3 * k + 2]} * ri;
    bool buried = false;
    for (int j = 0; j < n_nb && !buried; ++j) {
      const D3 d = {t.x - w.nx[j], t.y - w.ny[j], t.z - w.nz[j]};
      buried = norm2(d) < w.nr2[j];
    }
    acc += buried ? 0 : 1;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(kFull, acc, o);
  if (lane == 0) {
    const double area = static_cast<double>(acc) / n_dots * 4.0 * kPi * ri * ri;
    a.area[i] = area;
    a.energy[i] = a.gamma[i] * area;
  }
}

constexpr size_t kWarpSmemBytes = sizeof(WarpSmem) * kWarps;

}  // namespace

cudaError_t sasa_prepare() {
  cudaError_t e = cudaFuncSetAttribute(k_sasa_boundary, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(kWarpSmemBytes));
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_sasa_areas, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              static_cast<int>(kWarpSmemBytes));
}

void launch_sasa_forces(const SasaArgs& a, cudaStream_t s) {
  if (a.n_tasks <= 0) return;
  cudaMemsetAsync(a.counts, 0, 2 * sizeof(int32_t), s);
  k_sasa_boundary<<<(a.n_tasks + kWarps - 1) / kWarps, kWarps * 32, kWarpSmemBytes, s>>>(a);
  k_sasa_terms<<<148 * 8, 128, 0, s>>>(a);
}

void launch_sasa_areas(const SasaArgs& a, cudaStream_t s) {
  if (a.n_tasks <= 0) return;
  k_sasa_areas<<<(a.n_tasks + kWarps - 1) / kWarps, kWarps * 32, kWarpSmemBytes, s>>>(a);
}

void launch_shrake_rupley(const SasaArgs& a, const double* dots, int n_dots, cudaStream_t s) {
  if (a.n_tasks <= 0) return;
  k_shrake_rupley<<<(a.n_tasks + kWarps - 1) / kWarps, kWarps * 32, 0, s>>>(a, dots, n_dots);
}

}  // namespace ogk
