// Geometry of the PowerSasa boundary and the reverse-mode gradient of its
// Gauss-Bonnet terms, shared by the device kernels (sasa.cu) and a CPU test
// shim (plain C++ when not compiled by nvcc).
//
// The reference differentiates the accessible area with forward-mode
// directional derivatives (crates/energy/src/powersasa/derivatives.rs:
// vertex_point_jvp :222, arc_theta_jvp :346, vertex_epsilon_jvp :466), one
// per (atom, axis).  Each arc term theta_e cos(alpha_K) and each vertex
// exterior angle epsilon_v depends on at most four atoms, so here each term
// is differentiated once in reverse mode with respect to all of their
// coordinates: the same derivatives (the JVPs are linear in the tangent),
// evaluated as one adjoint sweep per term instead of up to twelve tangents.
// Failure conditions (degenerate caps, parallel axes, empty intersections,
// zero-length projections) are the reference's and zero the same parts.
#pragma once

#include <cmath>

#if defined(__CUDACC__)
#define OG_HD __host__ __device__ __forceinline__
#else
#define OG_HD inline
#endif

namespace ogsasa {

struct D3 {
  double x, y, z;
};
OG_HD D3 operator+(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
OG_HD D3 operator-(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
OG_HD D3 operator*(D3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
OG_HD D3 operator/(D3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
OG_HD double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
OG_HD D3 cross(D3 a, D3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
OG_HD double norm2(D3 a) { return dot(a, a); }
OG_HD double norm(D3 a) { return sqrt(norm2(a)); }

// Cap of neighbour k on atom i's unit sphere as a function of the two
// centres: axis w = (p_k - p_i)/d, cos alpha = (d^2 + r_i^2 - r_k^2)/(2 d r_i)
// (arrangement.rs:69-97), and d(cos alpha)/dd (derivatives.rs:183).
struct CapG {
  D3 w;
  double c, d, dcos_dd;
};

OG_HD bool cap_from(D3 pi, D3 pk, double ri, double rk, CapG* cap) {
  const D3 r = pk - pi;
  const double d2 = norm2(r);
  const double d = sqrt(d2);
  if (d < 1e-12) return false;
  cap->w = r / d;
  cap->d = d;
  cap->c = (d2 + ri * ri - rk * rk) / (2.0 * d * ri);
  cap->dcos_dd = (d2 - ri * ri + rk * rk) / (2.0 * d2 * ri);
  return true;
}

// Adjoint of (w, c) -> gradient with respect to p_k (p_i receives the
// negative).
OG_HD D3 cap_adjoint(const CapG& cap, D3 wbar, double cbar) {
  return (wbar - cap.w * dot(cap.w, wbar)) / cap.d + cap.w * (cbar * cap.dcos_dd);
}

// Intersection point of the circles of caps (w1, c1) and (w2, c2) on the
// root `sign` (derivatives.rs:92 vertex_point), with the intermediates the
// adjoint needs.
struct VpState {
  D3 w1, w2, np, v;
  double c1, c2, sigma, den, a, b, c, mn;
  int sign;
};

OG_HD bool vp_forward(D3 w1, double c1, D3 w2, double c2, int sign, VpState* s) {
  const double sigma = dot(w1, w2);
  const double den = 1.0 - sigma * sigma;
  if (fabs(den) < 1e-12) return false;
  const double a = (c1 - sigma * c2) / den;
  const double b = (c2 - sigma * c1) / den;
  const double csq = 1.0 - a * a - b * b - 2.0 * a * b * sigma;
  if (csq <= 0.0) return false;
  const double c = sqrt(csq);
  const D3 m = cross(w1, w2);
  const double mn = norm(m);
  if (mn < 1e-12) return false;
  s->w1 = w1;
  s->w2 = w2;
  s->c1 = c1;
  s->c2 = c2;
  s->sigma = sigma;
  s->den = den;
  s->a = a;
  s->b = b;
  s->c = c;
  s->mn = mn;
  s->np = m / mn;
  s->sign = sign;
  s->v = w1 * a + w2 * b + s->np * (c * static_cast<double>(sign));
  return true;
}

// v-bar -> (w1-bar, w2-bar, c1-bar, c2-bar), accumulated.
OG_HD void vp_adjoint(const VpState& s, D3 vbar, D3* w1b, D3* w2b, double* c1b, double* c2b) {
  const double sg = static_cast<double>(s.sign);
  double abar = dot(vbar, s.w1);
  double bbar = dot(vbar, s.w2);
  D3 g1 = vbar * s.a;
  D3 g2 = vbar * s.b;
  const double cbar = sg * dot(vbar, s.np);
  const D3 npbar = vbar * (sg * s.c);
  const D3 mbar = (npbar - s.np * dot(s.np, npbar)) / s.mn;
  g1 = g1 + cross(s.w2, mbar);
  g2 = g2 + cross(mbar, s.w1);
  const double csqbar = cbar / (2.0 * s.c);
  abar += csqbar * (-2.0 * s.a - 2.0 * s.b * s.sigma);
  bbar += csqbar * (-2.0 * s.b - 2.0 * s.a * s.sigma);
  double sigbar = csqbar * (-2.0 * s.a * s.b);
  const double na = abar / s.den, nb = bbar / s.den;
  const double denbar = -(abar * s.a + bbar * s.b) / s.den;
  *c1b += na - nb * s.sigma;
  *c2b += nb - na * s.sigma;
  sigbar += -na * s.c2 - nb * s.c1 - 2.0 * s.sigma * denbar;
  *w1b = *w1b + g1 + s.w2 * sigbar;
  *w2b = *w2b + g2 + s.w1 * sigbar;
}

// u = (v - w (v.w)) / |v - w (v.w)| and its adjoint.
struct ProjState {
  D3 u;
  double n, vw;
};

OG_HD bool proj_forward(D3 v, D3 w, ProjState* s) {
  s->vw = dot(v, w);
  const D3 p = v - w * s->vw;
  s->n = norm(p);
  if (s->n < 1e-12) return false;
  s->u = p / s->n;
  return true;
}

OG_HD void proj_adjoint(const ProjState& s, D3 v, D3 w, D3 ubar, D3* vb, D3* wb) {
  const D3 pbar = (ubar - s.u * dot(s.u, ubar)) / s.n;
  const double wp = dot(w, pbar);
  *vb = *vb + pbar - w * wp;
  *wb = *wb - pbar * s.vw - v * wp;
}

// t = (v x w) / |v x w| and its adjoint.
struct TanState {
  D3 t;
  double n;
};

OG_HD bool tan_forward(D3 v, D3 w, TanState* s) {
  const D3 c = cross(v, w);
  s->n = norm(c);
  if (s->n < 1e-12) return false;
  s->t = c / s->n;
  return true;
}

OG_HD void tan_adjoint(const TanState& s, D3 v, D3 w, D3 tbar, D3* vb, D3* wb) {
  const D3 cbar = (tbar - s.t * dot(s.t, tbar)) / s.n;
  *vb = *vb + cross(w, cbar);
  *wb = *wb + cross(cbar, v);
}

// Gradient of one arc's Gauss-Bonnet term theta cos(alpha_k) with respect to
// the centres of atom i, the arc's cap owner k and the owners l, m of the
// other caps at its start and end vertices (roots ss, se), as the sum over
// atoms x of directional_area_derivative's arc part (analytical.rs:337-398):
// theta d(cos alpha_k) + cos(alpha_k) d(theta).  `vertexed` = false (a full
// circle or a vertex not found) keeps the first part only, as the reference
// does.  Accumulates into gi, gk, gl, gm.
OG_HD void arc_gradient(D3 pi, D3 pk, D3 pl, D3 pm, double ri, double rk, double rl, double rm, int ss, int se,
                        double theta, bool vertexed, D3* gi, D3* gk, D3* gl, D3* gm) {
  CapG ck;
  if (!cap_from(pi, pk, ri, rk, &ck)) return;  // cos_alpha_directional = 0, arc_theta_jvp fails
  D3 wkb = {0.0, 0.0, 0.0};
  double ckb = theta;  // theta * d(cos alpha_k)
  if (vertexed) {
    CapG cl, cm;
    VpState s, e;
    ProjState ps, pe;
    if (cap_from(pi, pl, ri, rl, &cl) && cap_from(pi, pm, ri, rm, &cm) &&
        vp_forward(ck.w, ck.c, cl.w, cl.c, ss, &s) && vp_forward(ck.w, ck.c, cm.w, cm.c, se, &e) &&
        proj_forward(s.v, ck.w, &ps) && proj_forward(e.v, ck.w, &pe)) {
      // d(theta) = cos_t d(sin_t) - sin_t d(cos_t), cos_t = us.ue,
      // sin_t = w_k.(us x ue); seeded with cos(alpha_k).
      const D3 us = ps.u, ue = pe.u;
      const D3 x = cross(us, ue);
      const double cos_t = dot(us, ue);
      const double sin_t = dot(ck.w, x);
      const double sinb = ck.c * cos_t, cosb = -ck.c * sin_t;
      wkb = wkb + x * sinb;
      const D3 xb = ck.w * sinb;
      const D3 usb = cross(ue, xb) + ue * cosb;
      const D3 ueb = cross(xb, us) + us * cosb;
      D3 vsb = {0.0, 0.0, 0.0}, veb = {0.0, 0.0, 0.0};
      proj_adjoint(ps, s.v, ck.w, usb, &vsb, &wkb);
      proj_adjoint(pe, e.v, ck.w, ueb, &veb, &wkb);
      D3 wlb = {0.0, 0.0, 0.0}, wmb = {0.0, 0.0, 0.0};
      double clb = 0.0, cmb = 0.0;
      vp_adjoint(s, vsb, &wkb, &wlb, &ckb, &clb);
      vp_adjoint(e, veb, &wkb, &wmb, &ckb, &cmb);
      const D3 gl_ = cap_adjoint(cl, wlb, clb);
      const D3 gm_ = cap_adjoint(cm, wmb, cmb);
      *gl = *gl + gl_;
      *gm = *gm + gm_;
      *gi = *gi - gl_ - gm_;
    }
  }
  const D3 gk_ = cap_adjoint(ck, wkb, ckb);
  *gk = *gk + gk_;
  *gi = *gi - gk_;
}

// Gradient of a vertex's exterior angle epsilon (vertex_epsilon_jvp,
// derivatives.rs:466) with respect to atom i and the owners k (incoming cap)
// and l (outgoing cap).  Accumulates into gi, gk, gl.
OG_HD void vertex_gradient(D3 pi, D3 pk, D3 pl, double ri, double rk, double rl, int sign, D3* gi, D3* gk,
                           D3* gl) {
  CapG ck, cl;
  VpState s;
  TanState ti, to;
  if (!cap_from(pi, pk, ri, rk, &ck) || !cap_from(pi, pl, ri, rl, &cl)) return;
  if (!vp_forward(ck.w, ck.c, cl.w, cl.c, sign, &s)) return;
  if (!tan_forward(s.v, ck.w, &ti) || !tan_forward(s.v, cl.w, &to)) return;
  const D3 x = cross(ti.t, to.t);
  const double cos_e = dot(ti.t, to.t);
  const double sin_e = dot(s.v, x);
  const double sinb = cos_e, cosb = -sin_e;
  D3 vb = x * sinb;
  const D3 xb = s.v * sinb;
  const D3 tib = cross(to.t, xb) + to.t * cosb;
  const D3 tob = cross(xb, ti.t) + ti.t * cosb;
  D3 wkb = {0.0, 0.0, 0.0}, wlb = {0.0, 0.0, 0.0};
  double ckb = 0.0, clb = 0.0;
  tan_adjoint(ti, s.v, ck.w, tib, &vb, &wkb);
  tan_adjoint(to, s.v, cl.w, tob, &vb, &wlb);
  vp_adjoint(s, vb, &wkb, &wlb, &ckb, &clb);
  const D3 gk_ = cap_adjoint(ck, wkb, ckb);
  const D3 gl_ = cap_adjoint(cl, wlb, clb);
  *gk = *gk + gk_;
  *gl = *gl + gl_;
  *gi = *gi - gk_ - gl_;
}

}  // namespace ogsasa
