// Test shim: exposes the product's reverse-mode PowerSasa term gradients
// (origami_b200/csrc/engine/sasa_geom.h, compiled here as plain C++) so the
// CPU tests can compare them with the oracle's directional derivatives.
#include "../origami_b200/csrc/engine/sasa_geom.h"

using ogsasa::D3;

static D3 at(const double* p, int k) { return {p[3 * k], p[3 * k + 1], p[3 * k + 2]}; }
static void put(double* g, int k, D3 v) {
  g[3 * k] = v.x;
  g[3 * k + 1] = v.y;
  g[3 * k + 2] = v.z;
}

extern "C" void shim_arc_gradient(const double* p, const double* r, int ss, int se, double theta, int vertexed,
                                  double* g) {
  D3 gi{0, 0, 0}, gk{0, 0, 0}, gl{0, 0, 0}, gm{0, 0, 0};
  ogsasa::arc_gradient(at(p, 0), at(p, 1), at(p, 2), at(p, 3), r[0], r[1], r[2], r[3], ss, se, theta, vertexed != 0,
                       &gi, &gk, &gl, &gm);
  put(g, 0, gi);
  put(g, 1, gk);
  put(g, 2, gl);
  put(g, 3, gm);
}

extern "C" void shim_vertex_gradient(const double* p, const double* r, int sign, double* g) {
  D3 gi{0, 0, 0}, gk{0, 0, 0}, gl{0, 0, 0};
  ogsasa::vertex_gradient(at(p, 0), at(p, 1), at(p, 2), r[0], r[1], r[2], sign, &gi, &gk, &gl);
  put(g, 0, gi);
  put(g, 1, gk);
  put(g, 2, gl);
}
