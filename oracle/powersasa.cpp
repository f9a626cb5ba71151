// ORACLE -- test infrastructure only.
//
// CPU FP64 restatement of origami's PowerSasa analytical SASA (Klenin et al.
// 2011 spherical Gauss-Bonnet) and its analytical gradient.  One extra entry
// point, orc_sasa_forces_tangent_one_root, applies the engine's deliberate
// change for tangent pairs (see build_atom_cache); orc_sasa_forces is the
// reference's rule.  Paths are
// relative to the reference's crates/energy/src/powersasa/ directory:
//   geometry.rs      SmallCircle, intersect_circles (:70-102), signed angles
//   arrangement.rs   build_caps (:69-97), find_boundary (:100-227),
//                    angular_position / sample_circle_point / midpoint_on_circle
//                    / wrap_2pi_positive / every_point_buried (:229-318),
//                    count_accessible_components (:327-391)
//   area.rs          bounded_area (:44-134), walk_faces_summing_vertices (:140-222)
//   derivatives.rs   vertex_point (:92), identify_root_sign (:117),
//                    cos_alpha_grad (:183), vertex_point_jvp (:222),
//                    arc_theta_jvp (:346), vertex_epsilon_jvp (:466)
//   analytical.rs    build_atom_cache (:101-214), atom_area_gradient (:285-311),
//                    directional_area_derivative (:315-421),
//                    add_sasa_forces_analytical (:583-649)
//   mod.rs           powersasa_energy (:55-111), radii / surface tension (:27-52)
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

namespace {

struct V3 {
  double x, y, z;
};
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator*(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 operator/(V3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double norm2(V3 a) { return dot(a, a); }
inline double norm(V3 a) { return std::sqrt(norm2(a)); }
inline V3 normalize(V3 a) { return a / norm(a); }
inline V3 P(const double* xyz, int i) { return {xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]}; }
constexpr double kPi = M_PI;

struct Cap {
  V3 axis;
  double cos_a;
};
Cap make_cap(V3 axis, double cos_a) { return {normalize(axis), cos_a}; }
double sin_alpha(Cap c) { return std::sqrt(std::max(1.0 - c.cos_a * c.cos_a, 0.0)); }
bool contains_strict(Cap c, V3 p) { return dot(p, c.axis) > c.cos_a + 1e-12; }

enum Isect { kTwo, kTangent, kDisjoint, kCoincident };

// geometry.rs:70-102
Isect intersect(Cap c1, Cap c2, V3* p, V3* q) {
  const double sigma = dot(c1.axis, c2.axis);
  const double denom = 1.0 - sigma * sigma;
  if (std::fabs(denom) < 1e-12) {
    return std::fabs(c1.cos_a - sigma * c2.cos_a) < 1e-9 ? kCoincident : kDisjoint;
  }
  const double a = (c1.cos_a - sigma * c2.cos_a) / denom;
  const double b = (c2.cos_a - sigma * c1.cos_a) / denom;
  const double c_sq = 1.0 - a * a - b * b - 2.0 * a * b * sigma;
  if (c_sq < -1e-9) return kDisjoint;
  const V3 base = c1.axis * a + c2.axis * b;
  if (std::fabs(c_sq) <= 1e-9) {
    *p = base;
    return kTangent;
  }
  const double c = std::sqrt(c_sq);
  const V3 nc = cross(c1.axis, c2.axis);
  const V3 off = (nc / norm(nc)) * c;
  *p = base + off;
  *q = base - off;
  return kTwo;
}

V3 helper_axis(V3 axis) {
  const double ax = std::fabs(axis.x), ay = std::fabs(axis.y), az = std::fabs(axis.z);
  if (ax < ay && ax < az) return {1.0, 0.0, 0.0};
  if (ay < az) return {0.0, 1.0, 0.0};
  return {0.0, 0.0, 1.0};
}

double angular_position(V3 point, Cap c) {
  const V3 h = helper_axis(c.axis);
  const V3 u = normalize(h - c.axis * dot(h, c.axis));
  const V3 v = cross(c.axis, u);
  const V3 proj = point - c.axis * dot(point, c.axis);
  return std::atan2(dot(proj, v), dot(proj, u));
}

V3 sample_circle_point(Cap c) {
  const V3 h = helper_axis(c.axis);
  const V3 perp = normalize(h - c.axis * dot(h, c.axis));
  return c.axis * c.cos_a + perp * sin_alpha(c);
}

V3 midpoint_on_circle(V3 point, Cap c, double delta) {
  const V3 axial = c.axis * dot(point, c.axis);
  const V3 radial = point - axial;
  const double rn = norm(radial);
  if (rn < 1e-12) return point;
  const V3 u = radial / rn;
  const V3 v = cross(c.axis, u);
  return axial + (u * std::cos(delta) + v * std::sin(delta)) * rn;
}

double wrap_2pi_positive(double t) {
  const double two_pi = 2.0 * kPi;
  while (t <= 0.0) t += two_pi;
  while (t > two_pi) t -= two_pi;
  return t;
}

bool every_point_buried(const std::vector<Cap>& caps) {
  for (int i = 0; i < 200; ++i) {
    const double phi = i * 0.39 + 0.1, theta = i * 0.71 + 0.2;
    const V3 p = normalize({std::sin(phi) * std::cos(theta), std::sin(phi) * std::sin(theta), std::cos(phi)});
    bool in_any = false;
    for (const Cap& c : caps)
      if (contains_strict(c, p)) { in_any = true; break; }
    if (!in_any) return false;
  }
  return true;
}

struct Arc {
  int cap;
  V3 start, end;
  double theta;
  bool full;
};
struct Vert {
  V3 point;
  int in_cap, out_cap;
};
enum Boundary { kExposed, kBuried, kBounded };

struct Trans {
  double angle;
  V3 p;
  int other;
};

// arrangement.rs:100-227
Boundary find_boundary(const std::vector<Cap>& caps, std::vector<Arc>* arcs, std::vector<Vert>* verts) {
  arcs->clear();
  verts->clear();
  if (caps.empty()) return kExposed;
  const int n = static_cast<int>(caps.size());
  std::vector<std::vector<Trans>> per(n);
  for (int k = 0; k < n; ++k) {
    for (int m = 0; m < n; ++m) {
      if (m == k) continue;
      V3 p, q;
      const Isect r = intersect(caps[k], caps[m], &p, &q);
      if (r == kTwo) {
        per[k].push_back({angular_position(p, caps[k]), p, m});
        per[k].push_back({angular_position(q, caps[k]), q, m});
      } else if (r == kTangent) {
        per[k].push_back({angular_position(p, caps[k]), p, m});
      }
    }
    std::stable_sort(per[k].begin(), per[k].end(), [](const Trans& a, const Trans& b) { return a.angle < b.angle; });
    std::vector<Trans> ded;
    for (const Trans& t : per[k])
      if (ded.empty() || norm2(t.p - ded.back().p) >= 1e-12) ded.push_back(t);
    per[k].swap(ded);
  }
  for (int k = 0; k < n; ++k) {
    const auto& vs = per[k];
    if (vs.empty()) {
      const V3 probe = sample_circle_point(caps[k]);
      bool buried = false;
      for (int m = 0; m < n; ++m)
        if (m != k && contains_strict(caps[m], probe)) { buried = true; break; }
      if (!buried) arcs->push_back({k, probe, probe, -2.0 * kPi, true});
      continue;
    }
    const int m = static_cast<int>(vs.size());
    for (int i = 0; i < m; ++i) {
      const Trans& a = vs[i];
      const Trans& b = vs[(i + 1) % m];
      const double ccw = wrap_2pi_positive(b.angle - a.angle);
      if (ccw < 1e-9) continue;
      const V3 mid = midpoint_on_circle(a.p, caps[k], ccw / 2.0);
      bool ok = true;
      for (int idx = 0; idx < n; ++idx)
        if (idx != k && contains_strict(caps[idx], mid)) { ok = false; break; }
      if (!ok) continue;
      arcs->push_back({k, b.p, a.p, -ccw, false});
      verts->push_back({a.p, k, a.other});
    }
  }
  if (arcs->empty() && every_point_buried(caps)) return kBuried;
  return kBounded;
}

// arrangement.rs:69-97.  Returns false when atom i is inside a neighbour.
bool build_caps(V3 pi, double ri, const std::vector<int>& nb, const double* xyz, const double* radii,
                std::vector<Cap>* caps, std::vector<int>* owners) {
  caps->clear();
  owners->clear();
  for (int j : nb) {
    const V3 pj = P(xyz, j);
    const double rj = radii[j];
    const double d = norm(pj - pi);
    if (d + ri <= rj) return false;
    if (d + rj <= ri || d >= ri + rj) continue;
    const V3 axis = (pj - pi) / d;
    const double cos_a = (d * d + ri * ri - rj * rj) / (2.0 * d * ri);
    if (!(cos_a >= -1.0 && cos_a <= 1.0)) continue;
    caps->push_back({axis, cos_a});
    owners->push_back(j);
  }
  return true;
}

// ---------------------------------------------------------------- area
int count_accessible_components(const std::vector<Cap>& caps) {
  if (caps.empty()) return 1;
  const int N = 500;
  std::vector<V3> probes(N);
  const double golden = kPi * (3.0 - std::sqrt(5.0));
  for (int i = 0; i < N; ++i) {
    const double z = 1.0 - (2.0 * i + 1.0) / N;
    const double r = std::sqrt(std::max(1.0 - z * z, 0.0));
    const double th = golden * i;
    probes[i] = {r * std::cos(th), r * std::sin(th), z};
  }
  std::vector<char> acc(N);
  bool any = false;
  for (int i = 0; i < N; ++i) {
    bool in_any = false;
    for (const Cap& c : caps)
      if (contains_strict(c, probes[i])) { in_any = true; break; }
    acc[i] = !in_any;
    any = any || acc[i];
  }
  if (!any) return 0;
  const double spacing = std::sqrt(4.0 * kPi / N);
  const double cos_thresh = std::cos(std::min(2.5 * spacing, kPi));
  std::vector<int> parent(N);
  for (int i = 0; i < N; ++i) parent[i] = i;
  auto root = [&](int x) {
    while (parent[x] != x) {
      parent[x] = parent[parent[x]];
      x = parent[x];
    }
    return x;
  };
  for (int i = 0; i < N; ++i) {
    if (!acc[i]) continue;
    for (int j = i + 1; j < N; ++j) {
      if (!acc[j]) continue;
      if (dot(probes[i], probes[j]) > cos_thresh) {
        const int ri = root(i), rj = root(j);
        if (ri != rj) parent[ri] = rj;
      }
    }
  }
  std::vector<int> roots;
  for (int i = 0; i < N; ++i)
    if (acc[i]) {
      const int r = root(i);
      if (std::find(roots.begin(), roots.end(), r) == roots.end()) roots.push_back(r);
    }
  return static_cast<int>(roots.size());
}

// area.rs:140-222
void walk_faces(const std::vector<Arc>& arcs, const std::vector<Cap>& caps, int* loops_out, double* vsum_out) {
  const int n = static_cast<int>(arcs.size());
  std::vector<char> visited(n, 0);
  int loops = 0;
  double vsum = 0.0;
  const double two_pi = 2.0 * kPi;
  for (int start = 0; start < n; ++start) {
    if (visited[start]) continue;
    if (arcs[start].full) {
      visited[start] = 1;
      ++loops;
      continue;
    }
    int current = start;
    // A well-formed loop returns to `start` within n steps; the reference
    // has no bound here (a cycle that misses `start` would not end), so
    // the walk stops after n steps, which changes nothing for well-formed
    // boundaries.
    for (int guard = 0; guard <= n; ++guard) {
      visited[current] = 1;
      const V3 end_pt = arcs[current].end;
      const V3 t_in = normalize(cross(end_pt, caps[arcs[current].cap].axis));
      std::vector<int> cands;
      for (int i = 0; i < n; ++i)
        if (!arcs[i].full && norm2(arcs[i].start - end_pt) < 1e-10) cands.push_back(i);
      if (cands.empty()) break;
      int best = cands[0];
      double best_angle = INFINITY;
      for (int c : cands) {
        if (c == current) continue;
        const V3 t_out = normalize(cross(end_pt, caps[arcs[c].cap].axis));
        double d = dot(t_in, t_out);
        d = std::min(std::max(d, -1.0), 1.0);
        double ang = std::atan2(dot(end_pt, cross(t_in, t_out)), d);
        if (ang <= 1e-9) ang += two_pi;
        if (ang < best_angle) {
          best_angle = ang;
          best = c;
        }
      }
      const V3 t_out = normalize(cross(end_pt, caps[arcs[best].cap].axis));
      double d = dot(t_in, t_out);
      d = std::min(std::max(d, -1.0), 1.0);
      vsum += std::atan2(dot(end_pt, cross(t_in, t_out)), d);
      if (best == start) break;
      current = best;
    }
    ++loops;
  }
  *loops_out = loops;
  *vsum_out = vsum;
}

// area.rs:44-134 (with the component count computed here)
double bounded_area(double radius, const std::vector<Cap>& caps, const std::vector<Arc>& arcs) {
  const double r_sq = radius * radius;
  const double four_pi_r2 = 4.0 * kPi * r_sq;
  if (arcs.empty()) return 0.0;
  int l;
  double vsum;
  walk_faces(arcs, caps, &l, &vsum);
  if (l == 0) return 0.0;
  double arc_sum = 0.0;
  for (const Arc& a : arcs) arc_sum += caps[a.cap].cos_a * a.theta;
  const int c = std::max(std::min(count_accessible_components(caps), l), 1);
  const int chi = 2 * c - l;
  const double area = r_sq * (2.0 * kPi * chi - arc_sum - vsum);
  return std::min(std::max(area, 0.0), four_pi_r2);
}

// -------------------------------------------------------------- derivatives
enum Sign { kPlus = 1, kMinus = -1 };

bool vertex_point(Cap c1, Cap c2, int sign, V3* out) {
  const double sigma = dot(c1.axis, c2.axis);
  const double denom = 1.0 - sigma * sigma;
  if (std::fabs(denom) < 1e-12) return false;
  const double a = (c1.cos_a - sigma * c2.cos_a) / denom;
  const double b = (c2.cos_a - sigma * c1.cos_a) / denom;
  const double c_sq = 1.0 - a * a - b * b - 2.0 * a * b * sigma;
  if (c_sq <= 0.0) return false;
  const V3 base = c1.axis * a + c2.axis * b;
  const V3 nc = cross(c1.axis, c2.axis);
  const double nn = norm(nc);
  if (nn < 1e-12) return false;
  *out = base + (nc / nn * std::sqrt(c_sq)) * static_cast<double>(sign);
  return true;
}

int identify_root_sign(Cap c1, Cap c2, V3 ref) {
  V3 vp, vm;
  if (!vertex_point(c1, c2, kPlus, &vp) || !vertex_point(c1, c2, kMinus, &vm)) return kPlus;
  return norm2(vp - ref) <= norm2(vm - ref) ? kPlus : kMinus;
}

double cos_alpha_directional(V3 pi, V3 pk, double ri, double rk, V3 dri, V3 drk) {
  const V3 r = pk - pi;
  const double d2 = norm2(r);
  const double d = std::sqrt(d2);
  if (d < 1e-12) return 0.0;
  const V3 u = r / d;
  const double dcos_dd = (d2 - ri * ri + rk * rk) / (2.0 * d2 * ri);
  const V3 gk = u * dcos_dd;
  return dot(gk * -1.0, dri) + dot(gk, drk);
}

double cap_cos(V3 pi, V3 pk, double ri, double rk) {
  const double d = norm(pk - pi);
  return (d * d + ri * ri - rk * rk) / (2.0 * d * ri);
}

bool vertex_point_jvp(V3 pi, V3 pk, V3 pl, double ri, double rk, double rl, int sign, V3 dri, V3 drk, V3 drl,
                      V3* out) {
  const V3 rkv = pk - pi;
  const double dik = norm(rkv);
  if (dik < 1e-12) return false;
  const V3 wk = rkv / dik;
  const V3 rlv = pl - pi;
  const double dil = norm(rlv);
  if (dil < 1e-12) return false;
  const V3 wl = rlv / dil;
  const double cak = (dik * dik + ri * ri - rk * rk) / (2.0 * dik * ri);
  const double cal = (dil * dil + ri * ri - rl * rl) / (2.0 * dil * ri);
  const double sigma = dot(wk, wl);
  const double denom = 1.0 - sigma * sigma;
  if (std::fabs(denom) < 1e-12) return false;
  const double a = (cak - sigma * cal) / denom;
  const double b = (cal - sigma * cak) / denom;
  const double c_sq = 1.0 - a * a - b * b - 2.0 * a * b * sigma;
  if (c_sq <= 0.0) return false;
  const double c = std::sqrt(c_sq);
  const V3 m = cross(wk, wl);
  const double mn = std::sqrt(norm2(m));
  if (mn < 1e-12) return false;
  const V3 np = m / mn;
  const V3 dvk = drk - dri;
  const V3 dwk = (dvk - wk * dot(wk, dvk)) / dik;
  const V3 dvl = drl - dri;
  const V3 dwl = (dvl - wl * dot(wl, dvl)) / dil;
  const double dcos_k = cos_alpha_directional(pi, pk, ri, rk, dri, drk);
  const double dcos_l = cos_alpha_directional(pi, pl, ri, rl, dri, drl);
  const double dsig = dot(dwk, wl) + dot(wk, dwl);
  const double dden = -2.0 * sigma * dsig;
  const double num_a = cak - sigma * cal;
  const double dnum_a = dcos_k - dsig * cal - sigma * dcos_l;
  const double da = (dnum_a * denom - num_a * dden) / (denom * denom);
  const double num_b = cal - sigma * cak;
  const double dnum_b = dcos_l - dsig * cak - sigma * dcos_k;
  const double db = (dnum_b * denom - num_b * dden) / (denom * denom);
  const double dcsq = -2.0 * a * da - 2.0 * b * db - 2.0 * (da * b + a * db) * sigma - 2.0 * a * b * dsig;
  const double dc = dcsq / (2.0 * c);
  const V3 dbase = wk * da + dwk * a + wl * db + dwl * b;
  const V3 dm = cross(dwk, wl) + cross(wk, dwl);
  const V3 dnp = (dm - np * dot(np, dm)) / mn;
  *out = dbase + (np * dc + dnp * c) * static_cast<double>(sign);
  return true;
}

bool project_unit(V3 v, V3 dv, V3 w, V3 dw, V3* u, V3* du) {
  const double vw = dot(v, w);
  const V3 proj = v - w * vw;
  const double dvw = dot(dv, w) + dot(v, dw);
  const V3 dproj = dv - dw * vw - w * dvw;
  const double n = norm(proj);
  if (n < 1e-12) return false;
  *u = proj / n;
  *du = (dproj - *u * dot(*u, dproj)) / n;
  return true;
}

bool arc_theta_jvp(V3 pi, V3 pk, V3 pl, V3 pm, double ri, double rk, double rl, double rm, int ss, int se, V3 dri,
                   V3 drk, V3 drl, V3 drm, double* out) {
  const V3 rkv = pk - pi;
  const double dik = norm(rkv);
  if (dik < 1e-12) return false;
  const V3 wk = rkv / dik;
  const V3 dv = drk - dri;
  const V3 dwk = (dv - wk * dot(wk, dv)) / dik;
  const double cak = (dik * dik + ri * ri - rk * rk) / (2.0 * dik * ri);
  const Cap ck = make_cap(wk, cak);
  const V3 rlv = pl - pi;
  const double dil = norm(rlv);
  if (dil < 1e-12) return false;
  const Cap cl = make_cap(rlv / dil, (dil * dil + ri * ri - rl * rl) / (2.0 * dil * ri));
  const V3 rmv = pm - pi;
  const double dim = norm(rmv);
  if (dim < 1e-12) return false;
  const Cap cm = make_cap(rmv / dim, (dim * dim + ri * ri - rm * rm) / (2.0 * dim * ri));
  V3 vs, ve, dvs, dve;
  if (!vertex_point(ck, cl, ss, &vs) || !vertex_point(ck, cm, se, &ve)) return false;
  if (!vertex_point_jvp(pi, pk, pl, ri, rk, rl, ss, dri, drk, drl, &dvs)) return false;
  if (!vertex_point_jvp(pi, pk, pm, ri, rk, rm, se, dri, drk, drm, &dve)) return false;
  V3 us, dus, ue, due;
  if (!project_unit(vs, dvs, wk, dwk, &us, &dus) || !project_unit(ve, dve, wk, dwk, &ue, &due)) return false;
  const double cos_t = dot(us, ue);
  const double dcos_t = dot(dus, ue) + dot(us, due);
  const V3 x = cross(us, ue);
  const double sin_t = dot(wk, x);
  const V3 dx = cross(dus, ue) + cross(us, due);
  const double dsin_t = dot(dwk, x) + dot(wk, dx);
  *out = cos_t * dsin_t - sin_t * dcos_t;
  return true;
}

bool make_tangent(V3 v, V3 dv, V3 w, V3 dw, V3* u, V3* du) {
  const V3 c = cross(v, w);
  const double n = norm(c);
  if (n < 1e-12) return false;
  *u = c / n;
  const V3 dc = cross(dv, w) + cross(v, dw);
  *du = (dc - *u * dot(*u, dc)) / n;
  return true;
}

bool vertex_epsilon_jvp(V3 pi, V3 pk, V3 pl, double ri, double rk, double rl, int sign, V3 dri, V3 drk, V3 drl,
                        double* out) {
  const V3 rkv = pk - pi;
  const double dik = norm(rkv);
  if (dik < 1e-12) return false;
  const V3 wk = rkv / dik;
  const V3 dvk = drk - dri;
  const V3 dwk = (dvk - wk * dot(wk, dvk)) / dik;
  const V3 rlv = pl - pi;
  const double dil = norm(rlv);
  if (dil < 1e-12) return false;
  const V3 wl = rlv / dil;
  const V3 dvl = drl - dri;
  const V3 dwl = (dvl - wl * dot(wl, dvl)) / dil;
  const double cak = (dik * dik + ri * ri - rk * rk) / (2.0 * dik * ri);
  const double cal = (dil * dil + ri * ri - rl * rl) / (2.0 * dil * ri);
  V3 v, dv;
  if (!vertex_point(make_cap(wk, cak), make_cap(wl, cal), sign, &v)) return false;
  if (!vertex_point_jvp(pi, pk, pl, ri, rk, rl, sign, dri, drk, drl, &dv)) return false;
  V3 tin, dtin, tout, dtout;
  if (!make_tangent(v, dv, wk, dwk, &tin, &dtin) || !make_tangent(v, dv, wl, dwl, &tout, &dtout)) return false;
  const double cos_e = dot(tin, tout);
  const double dcos_e = dot(dtin, tout) + dot(tin, dtout);
  const V3 x = cross(tin, tout);
  const double sin_e = dot(v, x);
  const V3 dx = cross(dtin, tout) + cross(tin, dtout);
  const double dsin_e = dot(dv, x) + dot(v, dx);
  *out = cos_e * dsin_e - sin_e * dcos_e;
  return true;
}

// ------------------------------------------------------------ atom cache
struct CArc {
  int cap, vs, ve;
  double theta;
  bool full;
};
struct CVert {
  int in_cap, out_cap, sign;
};

// analytical.rs:101-214 (without the loop / component counts, which the
// gradient does not use).  Returns false when the atom has no boundary.
// tangent_one_root = false is the reference (each vertex's root by
// proximity); true gives both vertices of a tangent pair the root
// s = +1 for the lower cap index and -1 for the higher, the engine's rule.
bool build_atom_cache(int i, const double* xyz, const double* radii, const std::vector<int>& cand,
                      std::vector<int>* owners, std::vector<CArc>* carcs, std::vector<CVert>* cverts,
                      bool tangent_one_root = false) {
  const V3 pi = P(xyz, i);
  const double ri = radii[i];
  std::vector<int> nb;
  for (int j : cand)
    if (norm(P(xyz, j) - pi) <= ri + radii[j]) nb.push_back(j);
  std::vector<Cap> caps;
  if (!build_caps(pi, ri, nb, xyz, radii, &caps, owners)) return false;
  std::vector<Arc> arcs;
  std::vector<Vert> verts;
  const Boundary b = find_boundary(caps, &arcs, &verts);
  if (b != kBounded) return false;
  cverts->clear();
  for (const Vert& v : verts) {
    V3 tp, tq;
    const bool tangent =
        tangent_one_root && intersect(caps[v.in_cap], caps[v.out_cap], &tp, &tq) == kTangent;
    cverts->push_back({v.in_cap, v.out_cap,
                       tangent ? (v.in_cap < v.out_cap ? kPlus : kMinus)
                               : identify_root_sign(caps[v.in_cap], caps[v.out_cap], v.point)});
  }
  auto find_vertex = [&](V3 t) {
    for (size_t k = 0; k < verts.size(); ++k)
      if (norm2(verts[k].point - t) < 1e-10) return static_cast<int>(k);
    return -1;
  };
  carcs->clear();
  for (const Arc& a : arcs) {
    if (a.full) carcs->push_back({a.cap, -1, -1, a.theta, true});
    else carcs->push_back({a.cap, find_vertex(a.start), find_vertex(a.end), a.theta, false});
  }
  return !carcs->empty();
}

// analytical.rs:315-421
double directional_derivative(int i, const double* xyz, const double* radii, const std::vector<int>& owners,
                              const std::vector<CArc>& arcs, const std::vector<CVert>& verts, int x_atom, V3 basis) {
  const V3 zero{0.0, 0.0, 0.0};
  auto dr_of = [&](int y) { return y == x_atom ? basis : zero; };
  const V3 pi = P(xyz, i);
  const double ri = radii[i];
  const V3 dri = dr_of(i);
  double sum_arc = 0.0;
  for (const CArc& a : arcs) {
    const int k = owners[a.cap];
    const V3 pk = P(xyz, k);
    const double rk = radii[k];
    const V3 drk = dr_of(k);
    const double dcos = cos_alpha_directional(pi, pk, ri, rk, dri, drk);
    const double cak = cap_cos(pi, pk, ri, rk);
    if (a.full || a.vs < 0 || a.ve < 0 || a.vs >= static_cast<int>(verts.size()) ||
        a.ve >= static_cast<int>(verts.size())) {
      sum_arc += a.theta * dcos;
      continue;
    }
    const CVert vs = verts[a.vs], ve = verts[a.ve];
    const int vs_other = vs.in_cap == a.cap ? vs.out_cap : vs.in_cap;
    const int vs_sign = vs.in_cap == a.cap ? vs.sign : -vs.sign;
    const int ve_other = ve.in_cap == a.cap ? ve.out_cap : ve.in_cap;
    const int ve_sign = ve.in_cap == a.cap ? ve.sign : -ve.sign;
    const int l = owners[vs_other], m = owners[ve_other];
    double dtheta = 0.0;
    if (!arc_theta_jvp(pi, pk, P(xyz, l), P(xyz, m), ri, rk, radii[l], radii[m], vs_sign, ve_sign, dri, drk,
                       dr_of(l), dr_of(m), &dtheta))
      dtheta = 0.0;
    sum_arc += a.theta * dcos + cak * dtheta;
  }
  double sum_vert = 0.0;
  for (const CVert& v : verts) {
    const int ka = owners[v.in_cap], la = owners[v.out_cap];
    double de = 0.0;
    if (!vertex_epsilon_jvp(pi, P(xyz, ka), P(xyz, la), ri, radii[ka], radii[la], v.sign, dri, dr_of(ka),
                            dr_of(la), &de))
      de = 0.0;
    sum_vert += de;
  }
  return -sum_arc - sum_vert;
}

}  // namespace

extern "C" {

// SASA radius (vdW + 1.4 A probe, mod.rs:27-37) and surface tension
// (kJ/mol/A^2, mod.rs:42-52 times 4.184 times gamma_scale) of an element
// code (0 H, 1 C, 2 N, 3 O, 4 P, 5 S).
double orc_sasa_radius(int element) {
  static const double vdw[6] = {1.20, 1.70, 1.55, 1.52, 1.80, 1.80};
  return vdw[element] + 1.4;
}

double orc_sasa_gamma(int element, double gamma_scale) {
  return (element == 1 || element == 5) ? 0.005 * 4.184 * gamma_scale : 0.0;
}

// Per-atom accessible area (A^2), powersasa_energy (mod.rs:55-111).
void orc_sasa_areas(int n, const double* xyz, const double* radii, double* area) {
#pragma omp parallel for schedule(dynamic, 4)
  for (int i = 0; i < n; ++i) {
    std::vector<int> nb;
    const V3 pi = P(xyz, i);
    for (int j = 0; j < n; ++j)
      if (j != i && norm(P(xyz, j) - pi) <= radii[i] + radii[j]) nb.push_back(j);
    std::vector<Cap> caps;
    std::vector<int> owners;
    area[i] = 0.0;
    if (!build_caps(pi, radii[i], nb, xyz, radii, &caps, &owners)) continue;
    std::vector<Arc> arcs;
    std::vector<Vert> verts;
    const Boundary b = find_boundary(caps, &arcs, &verts);
    if (b == kExposed) area[i] = 4.0 * kPi * radii[i] * radii[i];
    else if (b == kBounded) area[i] = bounded_area(radii[i], caps, arcs);
  }
}

// Directional derivatives of single Gauss-Bonnet terms (the pieces
// directional_area_derivative sums, analytical.rs:337-421), one tangent per
// (role, axis).  p holds the centres of (i, k, l, m) or (i, k, l), r their
// radii; g receives 12 or 9 values, role-major.  The roles' atoms are taken
// distinct.
void orc_arc_term_jvps(const double* p, const double* r, int ss, int se, double theta, int vertexed, double* g) {
  const V3 pi = P(p, 0), pk = P(p, 1), pl = P(p, 2), pm = P(p, 3);
  for (int role = 0; role < 4; ++role) {
    for (int axis = 0; axis < 3; ++axis) {
      V3 t[4] = {};
      (axis == 0 ? t[role].x : axis == 1 ? t[role].y : t[role].z) = 1.0;
      const double dcos = cos_alpha_directional(pi, pk, r[0], r[1], t[0], t[1]);
      double term = theta * dcos;
      if (vertexed) {
        double dth = 0.0;
        if (!arc_theta_jvp(pi, pk, pl, pm, r[0], r[1], r[2], r[3], ss, se, t[0], t[1], t[2], t[3], &dth)) dth = 0.0;
        term += cap_cos(pi, pk, r[0], r[1]) * dth;
      }
      g[3 * role + axis] = term;
    }
  }
}

void orc_vertex_term_jvps(const double* p, const double* r, int sign, double* g) {
  const V3 pi = P(p, 0), pk = P(p, 1), pl = P(p, 2);
  for (int role = 0; role < 3; ++role) {
    for (int axis = 0; axis < 3; ++axis) {
      V3 t[3] = {};
      (axis == 0 ? t[role].x : axis == 1 ? t[role].y : t[role].z) = 1.0;
      double de = 0.0;
      if (!vertex_epsilon_jvp(pi, pk, pl, r[0], r[1], r[2], sign, t[0], t[1], t[2], &de)) de = 0.0;
      g[3 * role + axis] = de;
    }
  }
}

// Shrake-Rupley per-atom area (A^2) with n_dots Fibonacci test points per
// atom (crates/energy/src/sasa.rs:65-110, points :182-197): a point is
// buried when strictly inside another expanded sphere.
void orc_shrake_rupley_areas(int n, const double* xyz, const double* radii, int n_dots, double* area) {
  std::vector<V3> dots(n_dots);
  const double phi = kPi * (std::sqrt(3.0) + 1.0);
  for (int k = 0; k < n_dots; ++k) {
    const double y = 1.0 - 2.0 * k / (n_dots - 1.0);
    const double r = std::sqrt(1.0 - y * y);
    const double th = phi * k;
    dots[k] = {std::cos(th) * r, y, std::sin(th) * r};
  }
#pragma omp parallel for schedule(dynamic, 8)
  for (int i = 0; i < n; ++i) {
    const V3 pi = P(xyz, i);
    const double ri = radii[i];
    std::vector<int> nb;
    for (int j = 0; j < n; ++j)
      if (j != i && norm(P(xyz, j) - pi) <= ri + radii[j]) nb.push_back(j);
    int acc = 0;
    for (const V3& d : dots) {
      const V3 t = pi + d * ri;
      bool buried = false;
      for (int j : nb)
        if (norm2(t - P(xyz, j)) < radii[j] * radii[j]) { buried = true; break; }
      acc += buried ? 0 : 1;
    }
    area[i] = static_cast<double>(acc) / n_dots * 4.0 * kPi * ri * ri;
  }
}

}  // extern "C"

// SASA forces F_x -= gamma_i dA_i/dr_x (add_sasa_forces_analytical,
// analytical.rs:583-649); f is ADDED to.
void sasa_forces(int n, const double* xyz, const double* radii, const double* gamma, double* f,
                 bool tangent_one_root) {
  std::vector<double> acc(3 * static_cast<size_t>(n), 0.0);
#pragma omp parallel
  {
    std::vector<double> local(3 * static_cast<size_t>(n), 0.0);
#pragma omp for schedule(dynamic, 4)
    for (int i = 0; i < n; ++i) {
      if (gamma[i] == 0.0) continue;
      std::vector<int> cand;
      const V3 pi = P(xyz, i);
      for (int j = 0; j < n; ++j)
        if (j != i && norm(P(xyz, j) - pi) <= radii[i] + radii[j]) cand.push_back(j);
      std::vector<int> owners;
      std::vector<CArc> arcs;
      std::vector<CVert> verts;
      if (!build_atom_cache(i, xyz, radii, cand, &owners, &arcs, &verts, tangent_one_root)) continue;
      std::vector<int> affected{i};
      for (int o : owners)
        if (std::find(affected.begin(), affected.end(), o) == affected.end()) affected.push_back(o);
      const double r_sq = radii[i] * radii[i];
      for (int x : affected) {
        for (int axis = 0; axis < 3; ++axis) {
          V3 basis{0.0, 0.0, 0.0};
          (axis == 0 ? basis.x : axis == 1 ? basis.y : basis.z) = 1.0;
          const double d = directional_derivative(i, xyz, radii, owners, arcs, verts, x, basis);
          local[3 * x + axis] -= d * r_sq * gamma[i];
        }
      }
    }
#pragma omp critical
    for (size_t k = 0; k < acc.size(); ++k) acc[k] += local[k];
  }
  for (size_t k = 0; k < acc.size(); ++k) f[k] += acc[k];
}

extern "C" {

// The reference's forces.
void orc_sasa_forces(int n, const double* xyz, const double* radii, const double* gamma, double* f) {
  sasa_forces(n, xyz, radii, gamma, f, false);
}

// The same with the engine's rule for tangent pairs (both vertices on one
// root, which cancels the pair's 1/sqrt(c_sq) terms); equal to
// orc_sasa_forces wherever no pair is in the tangent band.
void orc_sasa_forces_tangent_one_root(int n, const double* xyz, const double* radii, const double* gamma,
                                      double* f) {
  sasa_forces(n, xyz, radii, gamma, f, true);
}

}  // extern "C"
