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
#include <algorithm>
#include <cstddef>
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
constexpr int kSasaBatch = 32;        // circles per arrangement batch
constexpr uint8_t kNoOther = 0xFF;    // pseudo entry of a transition-free circle
constexpr int32_t kContained = 1 << 16;  // circle inside a cap it does not cross
constexpr int32_t kCountMask = kContained - 1;
// crossing masks: one bit per live circle below kMaskCircles, bit 63 for
// kContained
constexpr int kMaskCircles = 56;
constexpr uint64_t kMaskContained = 1ull << 63;
constexpr double kPi = 3.14159265358979323846;

// Optional per-phase cycle counters of the boundary kernels (measurement
// builds only: -DOG_SASA_PHASE_CLOCKS=1).  Lane 0 of each warp accumulates
// clock64() differences per phase in registers and adds them to
// g_sasa_phase when its atom is done; og_sasa_phase_clocks reads them.
// Phases: 0 caps, 1 nested-cap cull, 2 pair counts, 3 batch set-up,
// 4 transitions, 5 rank sort, 6 walk over the sorted order (ties,
// duplicates, burial bookkeeping, toggle scan; de-duplication), 7 exposure and arcs, 8 vertex
// signs and links, 9 term records; sums of 10 caps, 11 live circles,
// 12 transitions, 13 atoms.
constexpr int kPhases = 14;
#ifdef OG_SASA_PHASE_CLOCKS
__device__ unsigned long long g_sasa_phase[kPhases];
__device__ __forceinline__ long long cycles() {
  long long v = 0;
#ifdef __CUDA_ARCH__
  asm volatile("mov.u64 %0, %%clock64;" : "=l"(v));
#endif
  return v;
}
struct PhaseClock {
  unsigned long long acc[kPhases];
  long long t;
  __device__ PhaseClock() : t(cycles()) {
    for (int k = 0; k < kPhases; ++k) acc[k] = 0;
  }
  __device__ __forceinline__ void mark(int id) {
    const long long n = cycles();
    acc[id] += static_cast<unsigned long long>(n - t);
    t = n;
  }
  __device__ __forceinline__ void count(int id, int v) { acc[id] += static_cast<unsigned long long>(v); }
  __device__ __forceinline__ void flush(int lane) {
    if (lane == 0)
      for (int k = 0; k < kPhases; ++k) atomicAdd(&g_sasa_phase[k], acc[k]);
  }
};
#else
struct PhaseClock {
  __device__ __forceinline__ void mark(int) {}
  __device__ __forceinline__ void count(int, int) {}
  __device__ __forceinline__ void flush(int) {}
};
#endif

__device__ __forceinline__ D3 normalize(D3 a) { return a / norm(a); }

struct Cap {
  D3 axis;
  double c;
};

__device__ __forceinline__ bool contains_strict(Cap c, D3 p) { return dot(p, c.axis) > c.c + 1e-12; }

// geometry.rs:70-102, restated.  Circle 1 (cap axis a1, cos c1) and circle 2
// meet where the line through base = a a1 + b a2 along a1 x a2 pierces the
// unit sphere, a = (c1 - sigma c2) / (1 - sigma^2), b = (c2 - sigma c1) /
// (1 - sigma^2), c_sq = 1 - a^2 - b^2 - 2ab sigma; none for c_sq < -1e-9,
// one (tangent) for |c_sq| <= 1e-9, none for parallel axes (1 - sigma^2 <
// 1e-12).  Since (1 - sigma^2) c_sq = nn = 1 - sigma^2 - c1^2 - c2^2 + 2 sigma
// c1 c2, the classification needs no division.  It is written with explicit
// round-to-nearest intrinsics, which the compiler neither contracts nor
// reorders, so the counting pass (each unordered pair once) and the writing
// pass (each ordered pair) classify every pair bit for bit alike.
struct PairClass {
  double sigma, denom;
  int count;  // transitions: 0, 1 (tangent) or 2
};

__device__ __forceinline__ PairClass classify(Cap c1, Cap c2) {
  PairClass r;
  r.sigma = __fma_rn(c1.axis.x, c2.axis.x, __fma_rn(c1.axis.y, c2.axis.y, __dmul_rn(c1.axis.z, c2.axis.z)));
  r.denom = __fma_rn(-r.sigma, r.sigma, 1.0);
  r.count = 0;
  if (fabs(r.denom) < 1e-12) return r;
  // every step is symmetric in the two caps, so (1, 2) and (2, 1) agree too
  const double t = __fma_rn(2.0 * r.sigma, __dmul_rn(c1.c, c2.c), r.denom);
  const double nn = __dsub_rn(t, __dadd_rn(__dmul_rn(c1.c, c1.c), __dmul_rn(c2.c, c2.c)));
  const double eps = 1e-9 * r.denom;
  r.count = nn > eps ? 2 : (nn >= -eps ? 1 : 0);
  return r;
}

// The transition points of a pair with count 1 or 2 (q only for 2).  For
// unit axes |a1 x a2|^2 = 1 - sigma^2 = denom, so one reciprocal square root
// of denom gives both 1 / denom and the normalisation of a1 x a2 (equal to
// the reference's division and norm up to rounding).  *rate_sk receives
// sqrt(c_sq denom) = |(a1 x a2) . (p - base)|, the crossing rate times the
// circle's sin(alpha) (0 for count 1).
__device__ __forceinline__ void transition_points(Cap c1, Cap c2, PairClass pc, D3* p, D3* q, double* rate_sk) {
  const double rd = rsqrt(pc.denom);
  const double inv = rd * rd;
  const double a = (c1.c - pc.sigma * c2.c) * inv;
  const double b = (c2.c - pc.sigma * c1.c) * inv;
  const D3 base = c1.axis * a + c2.axis * b;
  *rate_sk = 0.0;
  if (pc.count == 1) {
    *p = base;
    return;
  }
  const double c_sq = 1.0 - a * a - b * b - 2.0 * a * b * pc.sigma;
  const D3 nc = cross(c1.axis, c2.axis);
  const double root = sqrt(fmax(c_sq, 0.0));
  *rate_sk = root * (pc.denom * rd);
  const D3 off = nc * (root * rd);
  *p = base + off;
  *q = base - off;
}

__device__ __forceinline__ D3 helper_axis(D3 axis) {
  const double ax = fabs(axis.x), ay = fabs(axis.y), az = fabs(axis.z);
  if (ax < ay && ax < az) return {1.0, 0.0, 0.0};
  if (ay < az) return {0.0, 1.0, 0.0};
  return {0.0, 0.0, 1.0};
}

__device__ __noinline__ D3 sample_circle_point(Cap c) {
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

// The frame in which a circle's transitions are ordered: fu, fv span the
// circle's plane (scale-free; only the angle matters).
__device__ __forceinline__ void slot_frame(D3 axis, D3* fu, D3* fv) {
  const D3 h = helper_axis(axis);
  *fu = h - axis * dot(h, axis);
  *fv = cross(axis, *fu);
}

// Pseudo-angle of unit radial direction u in the frame (fu, fv), in [-2, 2].
__device__ __forceinline__ double slot_angle(D3 u, D3 fu, D3 fv) { return pseudo_angle(dot(u, fu), dot(u, fv)); }

// Sort key of transition slot sl: its pseudo-angle shifted to [0, 4] and
// quantised (quantum Q = 2^-19), the slot below it (ties of equal quanta in
// slot order).  The quantum is taken in FP32 from the FP64 coordinates
// (x, y) of the point in the circle's frame; converting x and y, |x| + |y|,
// the approximate quotient (2 ulp), 1 -+ r and the shift by 2 leave the
// shifted angle within E = 13 * 2^-24 of the FP64 pseudo-angle.  Keys whose
// quanta differ by 2 or more are more than Q apart, so their angles differ
// by more than Q - 2E > 0 in the same direction: they order as the FP64
// angles do.  Neighbours in key order whose quanta differ by at most 1 are
// found after the sort and their circle ordered again from the FP64 angles
// (ties: slot order).  7 slot bits for buffers of up to 128 slots, else 8;
// the quantum needs 22 bits.
template <int kTrans>
struct SlotKey {
  static constexpr int kShift = kTrans <= 128 ? 7 : 8;
  static constexpr float kScale = 524288.0f;  // 1 / Q = 2^19: 4 * 2^19 < 2^22 <= 2^(32 - kShift)
  static __device__ __forceinline__ uint32_t pack(float shifted, int sl) {
    const float q = fminf(fmaxf(shifted, 0.0f), 4.0f) * kScale;
    return (__float2uint_rz(q) << kShift) | static_cast<uint32_t>(sl);
  }
  // the key of the point with frame coordinates (x, y)
  static __device__ __forceinline__ uint32_t make(double x, double y, int sl) {
    const float xf = __double2float_rn(x), yf = __double2float_rn(y);
    const float d = fabsf(xf) + fabsf(yf);
    const float r = d > 0.0f ? __fdividef(xf, d) : 0.0f;
    return pack((y >= 0.0 ? 1.0f - r : r - 1.0f) + 2.0f, sl);
  }
};

// identify_root_sign (derivatives.rs:117).
__device__ int identify_root_sign(Cap c1, Cap c2, D3 ref) {
  ogsasa::VpState sp, sm;
  if (!ogsasa::vp_forward(c1.axis, c1.c, c2.axis, c2.c, 1, &sp) ||
      !ogsasa::vp_forward(c1.axis, c1.c, c2.axis, c2.c, -1, &sm))
    return 1;
  return norm2(sp.v - ref) <= norm2(sm.v - ref) ? 1 : -1;
}

// ------------------------------------------------------ per-warp storage
// Capacities: caps (neighbour spheres cutting atom i's sphere), transitions
// of one batch of circles, exposed arcs (and vertices).  Indices into caps
// and transitions are bytes, so both stay below 255 (0xFF marks a circle's
// pseudo entry).
template <int kCaps_, int kTrans_, int kArcs_>
struct WarpSmemT {
  static constexpr int kCaps = kCaps_, kTrans = kTrans_, kArcs = kArcs_;
  static_assert(kCaps <= 254 && kTrans <= 254, "byte-sized cap and transition indices");
  static_assert(kCaps / 2 >= kMaskCircles, "a crossing mask for every circle of mask mode");
  // caps (indices in neighbour order, i.e. ascending atom index)
  double cx[kCaps], cy[kCaps], cz[kCaps], cc[kCaps];
  int32_t owner[kCaps];
  uint8_t live[kCaps];
  // per live circle either its transitions (low 16 bits) and kContained,
  // or -- up to kMaskCircles live circles, no tangent pair -- the mask of
  // the live circles it crosses (bit lm) and kMaskContained
  union {
    int32_t tcnt[kCaps];
    uint64_t xmask[kCaps / 2];
  };
  // transitions of the batch of circles being processed: unit radial
  // direction, sort key (quantised angle over the slot, SlotKey), the other
  // cap, the batch circle, the sorted order and each entry's rank in it
  double tx[kTrans], ty[kTrans], tz[kTrans];
  uint32_t tkey[kTrans];
  uint8_t tother[kTrans];
  uint8_t tseg[kTrans];
  uint8_t torder[kTrans];
  uint8_t trank[kTrans];
  // a leaving crossing's entering partner (the other slot of its pair), or
  // kNoOther when the pair is not one clean enter/leave crossing
  uint8_t tpart[kTrans];
  // per batch circle: first entry, entries kept after de-duplication,
  // transition-free circles before it, sin(alpha) and 1 / sin(alpha)
  uint16_t sbeg[kSasaBatch + 1];
  uint8_t skept[kSasaBatch], zpre[kSasaBatch];
  double bsk[kSasaBatch], binv[kSasaBatch];
  // crossing toggle of each transition, the toggles up to it in angular
  // order, and per batch circle the mode (0: burial
  // depth by toggles, 1: explicit midpoint tests) and the depth before its
  // first transition
  int8_t ttog[kTrans], tdep[kTrans];
  int32_t bmode[kSasaBatch];
  int32_t bbase[kSasaBatch];
  // exposed arcs
  double a_theta[kArcs], a_sx[kArcs], a_sy[kArcs], a_sz[kArcs];
  uint8_t a_cap[kArcs], a_full[kArcs], a_vis[kArcs];
  int16_t a_own[kArcs], a_vs[kArcs], a_ve[kArcs];
  // vertices (one per arc that is not a full circle)
  double v_x[kArcs], v_y[kArcs], v_z[kArcs];
  uint8_t v_in[kArcs], v_out[kArcs];
  int8_t v_sign[kArcs];
};

// The boundary kernels' storage: four warps per block at the default
// capacities; atoms that exceed them are queued for one warp per block at
// the large ones.
using WarpSmem = WarpSmemT<kSasaMaxCaps, kSasaMaxTrans, kSasaMaxArcs>;
using WarpSmemBig = WarpSmemT<kSasaBigCaps, kSasaBigTrans, kSasaBigArcs>;

template <class W>
__device__ __forceinline__ Cap cap_at(const W& w, int k) { return {{w.cx[k], w.cy[k], w.cz[k]}, w.cc[k]}; }
__device__ __forceinline__ D3 pos(const SasaArgs& a, int j) { return {a.x[j], a.y[j], a.z[j]}; }
// Unit radial direction of transition s of the circle being processed.
template <class W>
__device__ __forceinline__ D3 tpoint(const W& w, int s) { return {w.tx[s], w.ty[s], w.tz[s]}; }

// Position of the n-th (0-based) set bit of mask, which has more than n.
__device__ __forceinline__ int nth_set_bit(unsigned mask, int n) {
  int pos = 0;
#pragma unroll
  for (int width = 16; width > 0; width >>= 1) {
    const int c = __popc(mask & ((1u << width) - 1u));
    if (n >= c) {
      n -= c;
      mask >>= width;
      pos += width;
    }
  }
  return pos;
}

// Transitions of live circle li (low 16 bits) and kContained: in mask mode
// every crossing pair has two transitions.
template <class W>
__device__ __forceinline__ int32_t circle_tally(const W& w, int li, bool masks) {
  if (!masks) return w.tcnt[li];
  const uint64_t mk = w.xmask[li];
  return 2 * __popcll(mk & ~kMaskContained) | ((mk & kMaskContained) ? kContained : 0);
}

// Sets bit b of circle li's crossing mask by a 32-bit atomic on the word
// holding it (little-endian halves), which shared memory does natively.
template <class W>
__device__ __forceinline__ void mask_or(W& w, int li, int b) {
  atomicOr(reinterpret_cast<unsigned*>(&w.xmask[li]) + (b >> 5), 1u << (b & 31));
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
__device__ __noinline__ bool segment_midpoint(D3 ua, D3 ub, Cap ck, double sk, bool single, D3* mid, double* cos_ccw,
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

// Rarely taken parts of the arrangement, kept out of line so that they do
// not weigh on the register allocation of the loops around them.
// The circles of `tied` (a bit per batch circle) ordered from the FP64
// angles of their transitions, ties in slot order.
template <class W>
__device__ __noinline__ void reorder_tied(W& w, unsigned tied, int b0, int lane) {
  while (tied) {
    const int j = __ffs(tied) - 1;
    tied &= tied - 1;
    const int sb = w.sbeg[j], se = w.sbeg[j + 1];
    D3 fu, fv;
    slot_frame(cap_at(w, w.live[b0 + j]).axis, &fu, &fv);
    for (int sl = sb + lane; sl < se; sl += 32) {
      const double as = slot_angle(tpoint(w, sl), fu, fv);
      int rank = 0;
      for (int t = sb; t < se; ++t) {
        const double at = slot_angle(tpoint(w, t), fu, fv);
        rank += (at < as || (at == as && t < sl)) ? 1 : 0;
      }
      rank = min(rank, se - sb - 1);
      w.torder[sb + rank] = static_cast<uint8_t>(sl);
      w.trank[sl] = static_cast<uint8_t>(rank);
    }
  }
}

// Consecutive duplicates dropped from each batch circle's sorted order
// (|dp|^2 < 1e-12 against the last kept entry), one lane.
template <class W>
__device__ __noinline__ void compact_duplicates(W& w, int nb) {
  for (int j = 0; j < nb; ++j) {
    const int sb = w.sbeg[j], se = w.sbeg[j + 1];
    const double sk2 = w.bsk[j] * w.bsk[j];
    int kept = 0;
    for (int r = sb; r < se; ++r) {
      const int sl = w.torder[r];
      if (kept == 0 || norm2(tpoint(w, sl) - tpoint(w, w.torder[sb + kept - 1])) * sk2 >= 1e-12)
        w.torder[sb + kept++] = static_cast<uint8_t>(sl);
    }
    w.skept[j] = static_cast<uint8_t>(kept);
  }
}

// Builds caps and the exposed boundary of atom i in w.  Returns the outcome;
// for kBounded, *n_arcs / *n_verts are the boundary sizes (possibly zero).
template <class W>
__device__ int build_boundary(const SasaArgs& a, W& w, int i, int lane, int* n_arcs_out, int* n_verts_out,
                              int* n_live_out, PhaseClock& ph) {
  const int sys = a.atom_sys[i];
  const D3 pi = pos(a, i);
  const double ri = a.radius[i];
  const double half_inv_ri = 0.5 / ri;
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
    // the atoms of two hit tiles per trip (independent loads in flight); the
    // caps are written in ascending atom order, the first tile's first
    struct Nb {
      double x, y, z, r;
      bool ok;
    };
    auto load = [&](int j) {
      return Nb{a.x[j], a.y[j], a.z[j], a.radius[j], j != i && a.atom_sys[j] >= 0};
    };
    auto probe = [&](const Nb& n, double* ax, double* ay, double* az, double* ca) {
      if (!n.ok) return false;
      const double dx = n.x - pi.x, dy = n.y - pi.y, dz = n.z - pi.z;
      const double rj = n.r;
      // d and 1/d from one reciprocal square root (d = 0 exactly for
      // coincident centres); the quotients by d as products
      const double d2 = dx * dx + dy * dy + dz * dz;
      const double inv_d = rsqrt(d2);
      const double d = d2 > 0.0 ? d2 * inv_d : 0.0;
      if (d > ri + rj) return false;
      if (d + ri <= rj) {
        enclosed = true;
        return false;
      }
      if (d + rj <= ri || d >= ri + rj) return false;
      *ca = (d2 + ri * ri - rj * rj) * (inv_d * half_inv_ri);
      if (!(*ca >= -1.0 && *ca <= 1.0)) return false;
      *ax = dx * inv_d;
      *ay = dy * inv_d;
      *az = dz * inv_d;
      return true;
    };
    auto put_cap = [&](bool is_cap, int j, double ax, double ay, double az, double ca) {
      const unsigned caps = __ballot_sync(kFull, is_cap);
      if (is_cap) {
        const int slot = n_caps + __popc(caps & ((1u << lane) - 1u));
        if (slot < W::kCaps) {
          w.cx[slot] = ax;
          w.cy[slot] = ay;
          w.cz[slot] = az;
          w.cc[slot] = ca;
          w.owner[slot] = j;
        }
      }
      n_caps += __popc(caps);
    };
    while (hits) {
      const int b = __ffs(hits) - 1;
      hits &= hits - 1;
      const int b2 = hits ? __ffs(hits) - 1 : -1;
      if (b2 >= 0) hits &= hits - 1;
      const int j = (st.x + t0 + b) * 32 + lane;
      const int j2 = (st.x + t0 + b2) * 32 + lane;
      double ax = 0.0, ay = 0.0, az = 0.0, ca = 0.0, ax2 = 0.0, ay2 = 0.0, az2 = 0.0, ca2 = 0.0;
      const Nb n1 = load(j), n2 = load(b2 >= 0 ? j2 : j);
      const bool c1 = probe(n1, &ax, &ay, &az, &ca);
      const bool c2 = b2 >= 0 && probe(n2, &ax2, &ay2, &az2, &ca2);
      put_cap(c1, j, ax, ay, az, ca);
      if (b2 >= 0) put_cap(c2, j2, ax2, ay2, az2, ca2);
    }
  }
  ph.mark(0);
  ph.count(10, n_caps);
  if (__any_sync(kFull, enclosed)) return kBuried;
  if (n_caps > W::kCaps) return kInvalid;
  if (n_caps == 0) return kExposed;
  __syncwarp();

  // ---- drop caps whose circle lies inside another cap: alpha_k < alpha_m
  // and angle(axis_k, axis_m) < alpha_m - alpha_k, i.e. sigma - c_k c_m -
  // margin > s_k s_m, compared squared (both sides positive)
  // Each lane tests two caps (k and k + 32) against the caps m in one pass,
  // so a cap m's data is read once for both; survivors keep ascending order.
  int n_live = 0;
  for (int k0 = 0; k0 < n_caps; k0 += 64) {
    const int ka = k0 + lane, kb = k0 + 32 + lane;
    bool la = ka < n_caps, lb = kb < n_caps;
    const double ca = la ? w.cc[ka] : 0.0, cb = lb ? w.cc[kb] : 0.0;
    const double sa2 = 1.0 - ca * ca, sb2 = 1.0 - cb * cb;
    const D3 aa = la ? D3{w.cx[ka], w.cy[ka], w.cz[ka]} : D3{};
    const D3 ab = lb ? D3{w.cx[kb], w.cy[kb], w.cz[kb]} : D3{};
    for (int m = 0; m < n_caps && (la || lb); ++m) {
      const double cm = w.cc[m];
      const D3 am = {w.cx[m], w.cy[m], w.cz[m]};
      const double sm2 = 1.0 - cm * cm;
      if (la && m != ka && ca > cm) {
        const double lhs = dot(aa, am) - cm * ca - 1e-6;
        if (lhs > 0.0 && lhs * lhs > sa2 * sm2) la = false;
      }
      if (lb && m != kb && cb > cm) {
        const double lhs = dot(ab, am) - cm * cb - 1e-6;
        if (lhs > 0.0 && lhs * lhs > sb2 * sm2) lb = false;
      }
    }
    const unsigned below = (1u << lane) - 1u;
    const unsigned lva = __ballot_sync(kFull, la);
    if (la) w.live[n_live + __popc(lva & below)] = static_cast<uint8_t>(ka);
    n_live += __popc(lva);
    const unsigned lvb = __ballot_sync(kFull, lb);
    if (lb) w.live[n_live + __popc(lvb & below)] = static_cast<uint8_t>(kb);
    n_live += __popc(lvb);
  }
  __syncwarp();
  ph.mark(1);
  ph.count(11, n_live);

  // ---- boundary arcs (find_boundary), a batch of circles at a time: the
  // transitions of every circle are counted first (each ordered pair once,
  // by the same classification the writing pass uses), then consecutive
  // circles whose transition lists fit the buffer are processed together --
  // their transitions written, sorted and tested across all lanes -- and the
  // exposed arcs appended in circle order and, within a circle, in angular
  // order, the reference's order.  A circle without transitions takes one
  // pseudo entry (its probe test).  A circle that lies inside a cap without
  // crossing its rim (possible only within the culling margin) is marked
  // kContained.  With at most kMaskCircles live circles the pass records
  // which circles cross (masks), so that the writing pass visits only
  // crossing pairs; a tangent pair (one transition) sends the atom back to
  // plain counts.
  // p / n_live by a float reciprocal: exact here, since p + 0.5 keeps the
  // quotient at least 0.5 / n_live from an integer, far above the rounding
  const float inv_live = 1.0f / static_cast<float>(n_live);
  bool masks = n_live <= kMaskCircles;
  for (int pass = 0; pass < 2; ++pass) {
    if (masks) {
      for (int li = lane; li < n_live; li += 32) w.xmask[li] = 0;
    } else {
      for (int li = lane; li < n_live; li += 32) w.tcnt[li] = 0;
    }
    __syncwarp();
    // the counts are symmetric (circle k crosses cap m where circle m
    // crosses cap k), so each unordered pair is classified once: pair p of
    // the n(n-1)/2 with li < lm, row-major.  Row l starts at
    // S(l) = l (2n - 1 - l) / 2; the row of p is the floor of the smaller
    // root of S(l) = p, corrected by one step for the rounding of sqrtf
    // (the discriminant is an exact float: below 2^24).
    const int n_pairs = n_live * (n_live - 1) / 2;
    const float tn = static_cast<float>(2 * n_live - 1);
    bool tangent = false;
    for (int p = lane; p < n_pairs; p += 32) {
      int li = static_cast<int>((tn - sqrtf(tn * tn - 8.0f * static_cast<float>(p))) * 0.5f);
      li = max(0, min(li, n_live - 2));
      if ((li + 1) * (2 * n_live - 2 - li) / 2 <= p) {
        ++li;
      } else if (li * (2 * n_live - 1 - li) / 2 > p) {
        --li;
      }
      const int lm = li + 1 + p - li * (2 * n_live - 1 - li) / 2;
      const Cap ck = cap_at(w, w.live[li]), cm = cap_at(w, w.live[lm]);
      const PairClass pc = classify(ck, cm);
      // a circle inside the other cap without crossing its rim
      const bool in_m = !pc.count && ck.c * pc.sigma - cm.c > -1e-9;
      const bool in_k = !pc.count && cm.c * pc.sigma - ck.c > -1e-9;
      if (masks) {
        tangent |= pc.count == 1;
        if (pc.count == 2) {
          mask_or(w, li, lm);
          mask_or(w, lm, li);
        }
        if (in_m) mask_or(w, li, 63);
        if (in_k) mask_or(w, lm, 63);
      } else {
        if (pc.count) {
          atomicAdd(&w.tcnt[li], pc.count);
          atomicAdd(&w.tcnt[lm], pc.count);
        }
        if (in_m) atomicOr(&w.tcnt[li], kContained);
        if (in_k) atomicOr(&w.tcnt[lm], kContained);
      }
    }
    __syncwarp();
    if (!masks || !__any_sync(kFull, tangent)) break;
    masks = false;
  }
  ph.mark(2);

  int n_arcs = 0, n_verts = 0;
  bool bad = false;
  for (int b0 = 0; b0 < n_live && !bad;) {
    // the batch: consecutive live circles whose (padded) lists fit.  Lane j
    // takes circle b0 + j (kSasaBatch == 32): an inclusive warp prefix of
    // the list sizes gives every circle's first slot, and the lanes whose
    // prefix fits the buffer form the batch (a leading run, since the prefix
    // grows with j).  (Lane 0 alone walking the circles took twice as long.)
    static_assert(kSasaBatch == 32, "one batch circle per lane");
    const int cj = b0 + lane;
    const int tally = cj < n_live ? circle_tally(w, cj, masks) : 0;
    const int cnt_j = tally & kCountMask;
    const int sz = cj < n_live ? max(cnt_j, 1) : 0;
    const int zero_j = (cj < n_live && cnt_j == 0) ? 1 : 0;
    int incl = sz, zincl = zero_j;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int v = __shfl_up_sync(kFull, incl, d), z = __shfl_up_sync(kFull, zincl, d);
      if (lane >= d) {
        incl += v;
        zincl += z;
      }
    }
    const int nb = __popc(__ballot_sync(kFull, cj < n_live && incl <= W::kTrans));
    if (nb == 0) {
      bad = true;  // one circle alone has more transitions than the buffer
      break;
    }
    const int b1 = b0 + nb;
    if (lane < nb) {
      w.sbeg[lane] = static_cast<uint16_t>(incl - sz);
      w.zpre[lane] = static_cast<uint8_t>(zincl - zero_j);
      const double c = w.cc[w.live[cj]];
      const double sk = sqrt(fmax(1.0 - c * c, 0.0));
      w.bsk[lane] = sk;
      w.binv[lane] = sk > 0.0 ? 1.0 / sk : 0.0;
      w.bmode[lane] = (tally & kContained) ? 1 : 0;
      w.bbase[lane] = 0;
    }
    if (lane == nb - 1) w.sbeg[nb] = static_cast<uint16_t>(incl);
    __syncwarp();
    ph.mark(3);

    // transitions: pairs (batch circle j, live circle m), j-major, m ascending
    // (the reference's push order), kept as unit radial directions u
    // (p = axis cos(alpha) + u sin(alpha)) with a pseudo-angle sort key.
    // In mask mode the crossing pairs are read from the masks.  Otherwise
    // pairs are classified 32 at a time; those that cross, with their
    // output positions, go to a warp queue (one entry per lane) whose full
    // rounds build the points with every lane busy.
    int run = 0;
    bool mismatch = false, nonfinite = false;
    using Key = SlotKey<W::kTrans>;
    // the transitions of batch circle j with cap m from slot base on
    // batch circle j's transitions on its crossing with cap m, the points
    // in the order of the pair (circle j, cap m), from slot base on
    // (the two slots of a pair unrolled side by side)
    // Crossing direction: moving counter-clockwise (along axis_k x u) the
    // point enters cap m where the rate (axis_k x u).axis_m is positive and
    // leaves it where negative; a tangent or a shallow crossing (|rate| <=
    // 1e-4) gets 0.  The rate is -u.(axis_k x axis_m), and with
    // u = (base - axis_k c_k +- (axis_k x axis_m) sqrt(c_sq)/sqrt(denom)) / sin(alpha)
    // and base in the plane of the two axes, it is -+ sqrt(c_sq denom) /
    // sin(alpha): p (the + root) leaves, q enters.
    auto put = [&](int j, int m, const Cap& ck, double rate_sk, int count, D3 pt, D3 qt, int base) {
      const int end = w.sbeg[j + 1];
      const double inv = w.binv[j];
      D3 fu, fv;
      slot_frame(ck.axis, &fu, &fv);
      const bool clean = count == 2 && rate_sk * inv > 1e-4;
      const int tg[2] = {clean ? -1 : 0, clean ? 1 : 0};
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int sl = base + e;
        if (e >= count || sl >= end) continue;  // sl >= end never expected: the counts agree
        const D3 u = ((e == 0 ? pt : qt) - ck.axis * ck.c) * inv;
        const double x = dot(u, fu), y = dot(u, fv);
        if (!isfinite(x) || !isfinite(y)) nonfinite = true;
        w.tkey[sl] = Key::make(x, y, sl);
        w.tx[sl] = u.x;
        w.ty[sl] = u.y;
        w.tz[sl] = u.z;
        w.tother[sl] = static_cast<uint8_t>(m);
        w.tseg[sl] = static_cast<uint8_t>(j);
        w.ttog[sl] = static_cast<int8_t>(tg[e]);
        // the leaving crossing's entering partner (read for leaving ones only)
        w.tpart[sl] = (e == 0 && clean) ? static_cast<uint8_t>(base + 1) : kNoOther;
      }
    };
    if (masks) {
      // the crossing pairs straight from the masks, 32 at a time: entry e
      // belongs to the batch circle whose inclusive prefix of crossing
      // partners first exceeds e, and is its r-th partner in ascending live
      // order, with slots sbeg[j] + 2r and + 2r + 1.  (Sharing one
      // intersection between the pairs (k, m) and (m, k) of two batch
      // circles was measured slower: the lane holding both does two
      // circles' slot work while the others wait.)
      const uint64_t mj = lane < nb ? (w.xmask[b0 + lane] & ~kMaskContained) : 0ull;
      int incl = __popcll(mj);
      for (int d = 1; d < 32; d <<= 1) {
        const int v = __shfl_up_sync(kFull, incl, d);
        if (lane >= d) incl += v;
      }
      const int n_ent = __shfl_sync(kFull, incl, 31);
      for (int e0 = 0; e0 < n_ent; e0 += 32) {
        const int e = e0 + lane;
        int j = 0;
#pragma unroll
        for (int step = 16; step > 0; step >>= 1) {
          if (__shfl_sync(kFull, incl, j + step - 1) <= e) j += step;
        }
        const uint64_t mk = __shfl_sync(kFull, mj, j);
        const int r = e - (__shfl_sync(kFull, incl, j) - __popcll(mk));
        if (e < n_ent) {
          const unsigned lo = static_cast<unsigned>(mk);
          const int clo = __popc(lo);
          const int lm = r < clo ? nth_set_bit(lo, r) : 32 + nth_set_bit(static_cast<unsigned>(mk >> 32), r - clo);
          const int m = w.live[lm];
          const Cap ck = cap_at(w, w.live[b0 + j]), cm = cap_at(w, m);
          const PairClass pc = classify(ck, cm);
          if (pc.count != 2) mismatch = true;  // never expected: classify is symmetric
          D3 pt{}, qt{};
          double rate_sk = 0.0;
          transition_points(ck, cm, pc, &pt, &qt, &rate_sk);
          put(j, m, ck, rate_sk, pc.count, pt, qt, w.sbeg[j] + 2 * r);
        }
      }
      run = 2 * n_ent;
    } else {
      int queued = 0;
      unsigned qentry = 0;  // pair index | output position << 16
      const int np = nb * n_live;
      auto drain = [&](int n_entries) {
        if (lane < n_entries) {
          const int pidx = static_cast<int>(qentry & 0xFFFFu), base = static_cast<int>(qentry >> 16);
          const int j = __float2int_rz((static_cast<float>(pidx) + 0.5f) * inv_live);
          const int m = w.live[pidx - j * n_live];
          const Cap ck = cap_at(w, w.live[b0 + j]), cm = cap_at(w, m);
          const PairClass pc = classify(ck, cm);
          D3 pt{}, qt{};
          double rate_sk = 0.0;
          transition_points(ck, cm, pc, &pt, &qt, &rate_sk);
          put(j, m, ck, rate_sk, pc.count, pt, qt, base);
        }
      };
      for (int p0 = 0; p0 < np; p0 += 32) {
        const int p = p0 + lane;
        int cnt = 0, j = 0;
        if (p < np) {
          j = __float2int_rz((static_cast<float>(p) + 0.5f) * inv_live);
          const int lm = p - j * n_live;
          const int k = w.live[b0 + j], m = w.live[lm];
          if (k != m) cnt = classify(cap_at(w, k), cap_at(w, m)).count;
        }
        // prefix of the counts (0, 1 or 2) from two ballots
        const unsigned c1 = __ballot_sync(kFull, cnt & 1), c2 = __ballot_sync(kFull, cnt & 2);
        const unsigned below = (1u << lane) - 1u;
        const int off = __popc(c1 & below) + 2 * __popc(c2 & below);
        const int tot = __popc(c1) + 2 * __popc(c2);
        const unsigned packed =
            static_cast<unsigned>(p) | (static_cast<unsigned>(run + off + (cnt ? w.zpre[j] : 0)) << 16);
        const unsigned crossing = __ballot_sync(kFull, cnt != 0);
        const int n_new = __popc(crossing);
        // lanes queued .. 31 take the first new entries
        int t = lane - queued;
        unsigned v = __shfl_sync(kFull, packed, (t >= 0 && t < n_new) ? nth_set_bit(crossing, t) : lane);
        if (t >= 0 && t < n_new) qentry = v;
        if (queued + n_new >= 32) {
          drain(32);
          // the rest start the next queue
          t = lane + (32 - queued);
          v = __shfl_sync(kFull, packed, t < n_new ? nth_set_bit(crossing, t) : lane);
          if (t < n_new) qentry = v;
          queued = queued + n_new - 32;
        } else {
          queued += n_new;
        }
        run += tot;
      }
      drain(queued);
    }
    if (__any_sync(kFull, mismatch || nonfinite)) {
      bad = true;
      break;
    }
    if (run + w.zpre[nb - 1] + ((circle_tally(w, b1 - 1, masks) & kCountMask) == 0 ? 1 : 0) != w.sbeg[nb]) {
      bad = true;  // the two passes disagree: never expected, but never written past
      break;
    }
    for (int j = lane; j < nb; j += 32) {
      if ((circle_tally(w, b0 + j, masks) & kCountMask) != 0) continue;
      const int sl = w.sbeg[j];
      w.tseg[sl] = static_cast<uint8_t>(j);
      w.tother[sl] = kNoOther;
      w.tkey[sl] = Key::pack(2.0f, sl);
      w.ttog[sl] = 0;
    }
    __syncwarp();
    const int n_tr = w.sbeg[nb];
    ph.mark(4);
    ph.count(12, n_tr);

    // stable sort of each circle's transitions by angle (ties: push order):
    // an entry's rank is the number of the circle's keys below its own.
    // (This replaced FP64 angle comparisons with slot tie-breaks, summing the
    // toggles on the way; four of those per trip with their loads issued
    // together had measured 1.8x slower.)
    constexpr int kShift = Key::kShift;
    for (int sl = lane; sl < n_tr; sl += 32) {
      const int j = w.tseg[sl];
      const int sb = w.sbeg[j], se = w.sbeg[j + 1];
      const uint32_t ks = w.tkey[sl];
      int rank = 0;
#pragma unroll 4
      for (int t = sb; t < se; ++t) rank += w.tkey[t] < ks ? 1 : 0;
      rank = min(rank, se - sb - 1);
      w.torder[sb + rank] = static_cast<uint8_t>(sl);
      w.trank[sl] = static_cast<uint8_t>(rank);
    }
    __syncwarp();
    ph.mark(5);
    // One walk over the sorted positions finds circles with neighbours in
    // key order less than two quanta apart, consecutive duplicates
    // (|dp|^2 < 1e-12 against the entry before; |dp| = sin(alpha) |du|; the
    // kept entries are picked below), and does the burial-depth bookkeeping:
    // a tangent or shallow crossing sends its circle to explicit tests, a
    // leaving crossing wraps around the start of the circle when its pair's
    // entering crossing -- the neighbouring slot of the same circle and cap
    // -- sorts after it, and a segmented inclusive scan of the toggles gives
    // the crossings up to and including each entry in angular order.  A
    // circle with such neighbours (rare: the quantum is 2^-21 of the angle's
    // range) is ordered again from the FP64 angles and the walk repeated.
    bool dup = false;
    for (int walk = 0; walk < 2; ++walk) {
      unsigned tied = 0;
      int carry = 0;
      dup = false;
      for (int r0 = 0; r0 < n_tr; r0 += 32) {
        const int r = r0 + lane;
        int sl = 0, v = 0;
        bool head = true;
        if (r < n_tr) {
          sl = w.torder[r];
          const int j = w.tseg[sl], sb = w.sbeg[j];
          head = r == sb;
          v = w.ttog[sl];
          if (!head) {
            const int pv = w.torder[r - 1];
            const uint32_t dq = (w.tkey[sl] >> kShift) - (w.tkey[pv] >> kShift);
            if (dq <= 1) tied |= 1u << j;
            // a duplicate is within (pi/2) 1e-6 / sin(alpha) of angle, so
            // within that many quanta (+2, the quantisation and the FP32
            // error); only those are measured
            const double sk = w.bsk[j];
            if (static_cast<double>(dq) * sk <= 2e-6 * Key::kScale + 2.0 &&
                norm2(tpoint(w, sl) - tpoint(w, pv)) * (sk * sk) < 1e-12) {
              dup = true;
              atomicOr(&w.bmode[j], 1);
            }
          }
          if (w.tother[sl] != kNoOther) {
            if (v == 0) {
              atomicOr(&w.bmode[j], 1);
            } else if (v == -1) {
              const int q = w.tpart[sl];
              if (q == kNoOther) {
                atomicOr(&w.bmode[j], 1);
              } else if (w.trank[q] > w.trank[sl]) {
                atomicAdd(&w.bbase[j], 1);
              }
            }
          }
        }
        if (lane == 0 && !head) v += carry;
        const unsigned heads = __ballot_sync(kFull, head) & ((2u << lane) - 1u);
        const int first = heads ? 31 - __clz(heads) : 0;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
          const int y = __shfl_up_sync(kFull, v, d);
          if (lane - d >= first) v += y;
        }
        if (r < n_tr) w.tdep[sl] = static_cast<int8_t>(v);
        carry = __shfl_sync(kFull, v, 31);
      }
      tied = __reduce_or_sync(kFull, tied);
      if (walk == 1 || tied == 0) break;
      // order the tied circles from the FP64 angles (ties: slot order) and
      // start the bookkeeping of the batch again
      __syncwarp();
      if (lane < nb) {
        w.bmode[lane] = (circle_tally(w, b0 + lane, masks) & kContained) ? 1 : 0;
        w.bbase[lane] = 0;
      }
      reorder_tied(w, tied, b0, lane);
      __syncwarp();
    }

    // Burial depth.  Along a circle whose crossings are all clean (no
    // tangent, no shallow crossing, nothing merged by de-duplication, no cap
    // holding it without a crossing), the point enters and leaves each
    // crossing cap once, so the depth just after a transition is the toggles
    // up to it plus the depth before the first transition -- the number of
    // caps whose leaving crossing comes before their entering one in angular
    // order, counted in the walk above.  A segment is exposed where the depth
    // is 0.  The other circles test every segment's midpoint against every
    // cap.
    __syncwarp();
    if (__any_sync(kFull, dup)) {
      if (lane == 0) compact_duplicates(w, nb);
    } else {
      for (int j = lane; j < nb; j += 32) w.skept[j] = static_cast<uint8_t>(w.sbeg[j + 1] - w.sbeg[j]);
    }
    __syncwarp();
    ph.mark(6);

    // exposure of every segment (and of every transition-free circle)
    for (int r0 = 0; r0 < n_tr; r0 += 32) {
      const int r = r0 + lane;
      bool exposed = false, full = false;
      double cos_ccw = 1.0, sin_ccw = 0.0;
      int sa = 0, sbn = 0, j = 0, k = 0;
      D3 probe{};
      if (r < n_tr) {
        const int jr = w.tseg[w.torder[r]];
        const int pos = r - w.sbeg[jr], kept = w.skept[jr];
        if (pos < kept) {
          j = jr;
          sa = w.torder[r];
          k = w.live[b0 + j];
          const int nxt = pos + 1 == kept ? 0 : pos + 1;
          if (w.tother[sa] == kNoOther) {
            // no transitions: exposed unless a probe on the circle is buried
            full = true;
            probe = sample_circle_point(cap_at(w, k));
            exposed = true;
            for (int lm = 0; lm < n_live && exposed; ++lm) {
              const int m = w.live[lm];
              if (m != k && contains_strict(cap_at(w, m), probe)) exposed = false;
            }
          } else if (w.bmode[j] == 0) {
            sbn = w.torder[w.sbeg[j] + nxt];
            if (w.bbase[j] + w.tdep[sa] == 0) {
              // the reference's skip of a vanishing segment (ccw < 1e-9)
              const D3 ua = tpoint(w, sa), ub = tpoint(w, sbn);
              cos_ccw = dot(ua, ub);
              sin_ccw = dot(D3{w.cx[k], w.cy[k], w.cz[k]}, cross(ua, ub));
              exposed = !(cos_ccw > 0.0 && sin_ccw >= 0.0 && sin_ccw < 2e-9 && atan2(sin_ccw, cos_ccw) < 1e-9);
            }
          } else {
            sbn = w.torder[w.sbeg[j] + nxt];
            const Cap ck = cap_at(w, k);
            D3 mid;
            if (segment_midpoint(tpoint(w, sa), tpoint(w, sbn), ck, w.bsk[j], kept == 1, &mid, &cos_ccw,
                                 &sin_ccw)) {
              // a buried segment usually lies in one of the two caps whose
              // circles bound it; testing those first ends most searches early
              exposed = !contains_strict(cap_at(w, w.tother[sa]), mid) &&
                        !contains_strict(cap_at(w, w.tother[sbn]), mid);
              for (int lm = 0; lm < n_live && exposed; ++lm) {
                const int m = w.live[lm];
                if (m != k && contains_strict(cap_at(w, m), mid)) exposed = false;
              }
            }
          }
        }
      }
      const unsigned ex = __ballot_sync(kFull, exposed);
      const unsigned exv = __ballot_sync(kFull, exposed && !full);
      if (n_arcs + __popc(ex) > W::kArcs) {
        bad = true;
        break;
      }
      if (exposed) {
        const unsigned below = (1u << lane) - 1u;
        const int e = n_arcs + __popc(ex & below);
        w.a_cap[e] = static_cast<uint8_t>(k);
        if (full) {
          w.a_full[e] = 1;
          w.a_theta[e] = -2.0 * kPi;
          w.a_sx[e] = probe.x;
          w.a_sy[e] = probe.y;
          w.a_sz[e] = probe.z;
          w.a_own[e] = -1;
        } else {
          const Cap ck = cap_at(w, k);
          const double sk = w.bsk[j];
          const int v = n_verts + __popc(exv & below);
          const D3 pb = circle_point(ck, sk, tpoint(w, sbn)), pa = circle_point(ck, sk, tpoint(w, sa));
          w.a_full[e] = 0;
          w.a_theta[e] = 0.0;  // the ccw angle, taken below for all arcs at once
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
      }
      n_arcs += __popc(ex);
      n_verts += __popc(exv);
    }
    __syncwarp();
    ph.mark(7);
    b0 = b1;
  }
  if (bad) return kInvalid;
  __syncwarp();
  // The arcs' ccw angles from their end points (the exposure rounds hold an
  // exposed segment or two each, so the arc tangents run side by side here
  // instead of one lane at a time there): the cosine and sine of the angle
  // from p_start - a c to p_end - a c about the axis, as segment_midpoint
  // takes them from the unit radial directions, up to a positive factor.
  for (int e = lane; e < n_arcs; e += 32) {
    if (w.a_full[e]) continue;
    const Cap ck = cap_at(w, w.a_cap[e]);
    const int v = w.a_own[e];
    const D3 c0 = ck.axis * ck.c;
    const D3 ua = D3{w.v_x[v], w.v_y[v], w.v_z[v]} - c0, ub = D3{w.a_sx[e], w.a_sy[e], w.a_sz[e]} - c0;
    double ccw = atan2(dot(ck.axis, cross(ua, ub)), dot(ua, ub));
    if (ccw <= 0.0) ccw += 2.0 * kPi;
    w.a_theta[e] = -ccw;
  }
  __syncwarp();
  *n_arcs_out = n_arcs;
  *n_verts_out = n_verts;
  *n_live_out = n_live;
  return kBounded;
}

// Vertex signs and arc->vertex links (build_atom_cache).
//
// A tangent pair (|c_sq| <= 1e-9: one transition, at the midpoint of the two
// roots) departs from the reference's proximity test on purpose.  Its vertex
// lies halfway between the roots, so proximity is decided by rounding, and
// each root's derivative carries a 1/sqrt(c_sq) term of opposite sign: the
// pair's two vertices, (k, m) and (m, k), cancel those terms only when they
// name the same root.  The root base + s c (a_k x a_m)/|a_k x a_m| of (k, m)
// is the root -s of (m, k), so s = +1 for the lower cap index and -1 for the
// higher one always names one root, and the gradient is then that of the
// area (a CH2 group whose two H caps just touch on the C sphere: 0.24
// kJ/mol/A by central differences of the area, ~9000 kJ/mol/A with the
// signs crossed).
template <class W>
__device__ void link_boundary(W& w, int n_arcs, int n_verts, int lane) {
  for (int v = lane; v < n_verts; v += 32) {
    const Cap ci = cap_at(w, w.v_in[v]), co = cap_at(w, w.v_out[v]);
    w.v_sign[v] = static_cast<int8_t>(classify(ci, co).count == 1
                                          ? (w.v_in[v] < w.v_out[v] ? 1 : -1)
                                          : identify_root_sign(ci, co, {w.v_x[v], w.v_y[v], w.v_z[v]}));
  }
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

// An atom whose arrangement exceeds the default capacities goes to the
// overflow queue (counts[2], overflow[]) for the large-capacity kernel; past
// the large capacities it is reported (kStatusSasaOverflow).
// Returns whether the atom was queued (warp-uniform).
__device__ __forceinline__ bool overflow_atom(const SasaArgs& a, int i, int sys, int lane, bool big) {
  int queued = 0;
  if (lane == 0) {
    if (!big) {
      const int q = atomicAdd(&a.counts[2], 1);
      if (q < a.overflow_cap) {
        a.overflow[q] = i;
        queued = 1;
      }
    }
    if (!queued) atomicOr(&a.sys[sys].status, kStatusSasaOverflow);
  }
  return __shfl_sync(kFull, queued, 0) != 0;
}

// Force path, stage 1: the boundary of atom i as term records
// (build_atom_cache + arc_other_cap_and_sign, analytical.rs:101-214, 655-670).
template <class W>
__device__ void boundary_task(const SasaArgs& a, W& w, int i, int lane, bool big) {
  const int sys = a.atom_sys[i];
  if (a.sys[sys].status & kStatusDiverged) return;
  int n_arcs = 0, n_verts = 0, n_live = 0;
  PhaseClock ph;
  ph.count(13, 1);
  const int outcome = build_boundary(a, w, i, lane, &n_arcs, &n_verts, &n_live, ph);
  if (outcome == kInvalid) {
    overflow_atom(a, i, sys, lane, big);
    ph.flush(lane);
    return;
  }
  if (outcome != kBounded || n_arcs == 0) {
    ph.flush(lane);
    return;
  }
  link_boundary(w, n_arcs, n_verts, lane);
  ph.mark(8);
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
  ph.mark(9);
  ph.flush(lane);
}

// Each warp takes atoms from the queue counts[3] until none are left (a
// persistent grid of resident blocks): atoms differ several-fold in work,
// and a warp whose atom was quick takes the next one instead of holding its
// slot until the slowest warp of its block is done.
__device__ __forceinline__ int next_task(const SasaArgs& a, int lane) {
  int task = 0;
  if (lane == 0) task = atomicAdd(&a.counts[3], 1);
  return __shfl_sync(kFull, task, 0);
}

__global__ void __launch_bounds__(kWarps * 32, 5) k_sasa_boundary(SasaArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  WarpSmem& w = reinterpret_cast<WarpSmem*>(smem_raw)[warp];
  for (int task = next_task(a, lane); task < a.n_tasks; task = next_task(a, lane))
    boundary_task(a, w, a.tasks[task], lane, false);
}

// The queued atoms, one warp per block at the large capacities (persistent:
// the queue length is known only on the device).
// (One-warp blocks leave registers to spare; the cap keeps the compiler from
// choosing a smaller allocation with spills.)
__global__ void __maxnreg__(168) k_sasa_boundary_big(SasaArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  WarpSmemBig& w = *reinterpret_cast<WarpSmemBig*>(smem_raw);
  const int n = min(a.counts[2], a.overflow_cap);
  for (int q = blockIdx.x; q < n; q += gridDim.x) boundary_task(a, w, a.overflow[q], threadIdx.x, true);
}

// Force path, stage 2: one term per thread, F_x += gamma_i R_i^2 dTerm/dr_x.
__global__ void __launch_bounds__(128, 4) k_sasa_terms(SasaArgs a) {
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
template <class W>
__device__ void walk_faces(W& w, int n_arcs, int lane, int* loops_out, double* vsum_out) {
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
template <class W>
__device__ int count_components(const SasaArgs& a, W& w, int n_live, int lane) {
  // labels over ty and tz (adjacent), acceptance flags over tx: the
  // transition arrays are free once the arrangement is done
  static_assert(offsetof(W, tz) == offsetof(W, ty) + sizeof(w.ty) &&
                    sizeof(w.ty) + sizeof(w.tz) >= kSasaProbes * sizeof(int16_t) && sizeof(w.tx) >= kSasaProbes,
                "probe scratch");
  volatile int16_t* lab = reinterpret_cast<int16_t*>(w.ty);
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

template <class W>
__device__ void areas_task(const SasaArgs& a, W& w, int i, int lane, bool big) {
  const int sys = a.atom_sys[i];
  const double ri = a.radius[i];
  const double four_pi_r2 = 4.0 * kPi * ri * ri;
  int n_arcs = 0, n_verts = 0, n_live = 0;
  PhaseClock ph;  // not flushed: the counters describe the force path
  const int outcome = build_boundary(a, w, i, lane, &n_arcs, &n_verts, &n_live, ph);
  double area = 0.0;
  if (outcome == kInvalid) {
    if (overflow_atom(a, i, sys, lane, big)) return;  // the large-capacity kernel writes its area
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

__global__ void __launch_bounds__(kWarps * 32, 5) k_sasa_areas(SasaArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  WarpSmem& w = reinterpret_cast<WarpSmem*>(smem_raw)[warp];
  for (int task = next_task(a, lane); task < a.n_tasks; task = next_task(a, lane))
    areas_task(a, w, a.tasks[task], lane, false);
}

__global__ void __launch_bounds__(32) k_sasa_areas_big(SasaArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  WarpSmemBig& w = *reinterpret_cast<WarpSmemBig*>(smem_raw);
  const int n = min(a.counts[2], a.overflow_cap);
  for (int q = blockIdx.x; q < n; q += gridDim.x) areas_task(a, w, a.overflow[q], threadIdx.x, true);
}

// Shrake-Rupley: one warp per atom, neighbours staged in shared memory,
// lanes over test points.
constexpr int kSrMaxNeighbours = 254;
struct SrSmem {
  double nx[kSrMaxNeighbours], ny[kSrMaxNeighbours], nz[kSrMaxNeighbours], nr2[kSrMaxNeighbours];
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
        if (slot < kSrMaxNeighbours) {
          w.nx[slot] = a.x[j];
          w.ny[slot] = a.y[j];
          w.nz[slot] = a.z[j];
          w.nr2[slot] = a.radius[j] * a.radius[j];
        }
      }
      n_nb += __popc(m);
    }
  }
  if (n_nb > kSrMaxNeighbours) {
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
constexpr size_t kBigSmemBytes = sizeof(WarpSmemBig);
constexpr int kBigGrid = 148 * 4;  // persistent one-warp blocks for the queue
// five resident CTAs per SM (228 KB, 1 KB reserved per CTA): 20 warps; at
// four (the capacities 128 caps, 128 transitions, 48 arcs) the kernel was
// 1.6 % slower
static_assert(5 * (kWarpSmemBytes + 1024) <= 228 * 1024, "boundary kernel no longer fits five CTAs per SM");

}  // namespace

cudaError_t sasa_prepare() {
  cudaError_t e = cudaFuncSetAttribute(k_sasa_boundary, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(kWarpSmemBytes));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_sasa_areas, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(kWarpSmemBytes));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_sasa_boundary_big, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(kBigSmemBytes));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_sasa_areas_big, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(kBigSmemBytes));
  return e;
}

// Resident blocks of a queue-driven kernel: the SM count times the blocks
// that fit (no more than the atoms need).
template <class K>
int resident_grid(K kernel, int n_tasks) {
  static int n_sm = 0;
  if (n_sm == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
  }
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kWarps * 32, kWarpSmemBytes);
  return std::max(1, std::min((n_tasks + kWarps - 1) / kWarps, std::max(per_sm, 1) * std::max(n_sm, 1)));
}

void launch_sasa_forces(const SasaArgs& a, cudaStream_t s) {
  if (a.n_tasks <= 0) return;
  cudaMemsetAsync(a.counts, 0, 4 * sizeof(int32_t), s);
  k_sasa_boundary<<<resident_grid(k_sasa_boundary, a.n_tasks), kWarps * 32, kWarpSmemBytes, s>>>(a);
  k_sasa_boundary_big<<<kBigGrid, 32, kBigSmemBytes, s>>>(a);
  k_sasa_terms<<<148 * 8, 128, 0, s>>>(a);
}

void launch_sasa_areas(const SasaArgs& a, cudaStream_t s) {
  if (a.n_tasks <= 0) return;
  cudaMemsetAsync(a.counts + 2, 0, 2 * sizeof(int32_t), s);
  k_sasa_areas<<<resident_grid(k_sasa_areas, a.n_tasks), kWarps * 32, kWarpSmemBytes, s>>>(a);
  k_sasa_areas_big<<<kBigGrid, 32, kBigSmemBytes, s>>>(a);
}

void launch_shrake_rupley(const SasaArgs& a, const double* dots, int n_dots, cudaStream_t s) {
  if (a.n_tasks <= 0) return;
  k_shrake_rupley<<<(a.n_tasks + kWarps - 1) / kWarps, kWarps * 32, 0, s>>>(a, dots, n_dots);
}

}  // namespace ogk

#ifdef OG_SASA_PHASE_CLOCKS
// Reads (and with reset != 0 clears) the phase counters of a measurement
// build; out receives kPhases values.
extern "C" int og_sasa_phase_clocks(unsigned long long* out, int reset) {
  if (cudaMemcpyFromSymbol(out, ogk::g_sasa_phase, sizeof(unsigned long long) * ogk::kPhases) != cudaSuccess)
    return 5;
  if (reset) {
    unsigned long long zero[ogk::kPhases] = {};
    if (cudaMemcpyToSymbol(ogk::g_sasa_phase, zero, sizeof(zero)) != cudaSuccess) return 5;
  }
  return 0;
}
#endif
