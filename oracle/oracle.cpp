// ORACLE -- test infrastructure only.
//
// A CPU FP64 restatement of origami's force, energy and integrator code, used
// by tests/ (as the checker), by __graft_entry__.smoke() and by bench.py's CPU
// baseline leg.  Nothing in the product (origami_b200/) links or calls it.
//
// Every function follows the reference file:line it cites (paths relative to
// the reference's crates/ directory).  Pair sums run over plain i<j loops with
// the same cutoff tests instead of origami's cell lists; that reorders the
// floating-point summation (the results agree to ~1e-15 relative), nothing
// else.  Pinned against origami's known answers in tests/test_oracle.py.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../include/origami_gpu.h"

namespace {

constexpr double kKcalToKj = 4.184;                 // energy/src/units.rs:4
constexpr double kCoulomb = 332.0637;               // energy/src/nonbonded.rs:34
constexpr double kEpsWater = 78.5;                  // energy/src/gb.rs:23
constexpr double kObcAlpha = 1.0, kObcBeta = 0.8, kObcGamma = 4.85;  // gb.rs:28-30
constexpr double kObcOffset = 0.09;                 // gb.rs:32
constexpr double kBoltzmann = 8.314462618e-3;       // dynamics/src/langevin.rs:44
constexpr double kAccel = 1.0e-4;                   // langevin.rs:47

double deg2rad(double d) { return d * M_PI / 180.0; }  // units.rs:13

struct V3 {
  double x, y, z;
};
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator*(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 operator/(V3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
inline V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double norm2(V3 a) { return dot(a, a); }
inline double norm(V3 a) { return std::sqrt(norm2(a)); }
inline V3 normalize(V3 a) { return a / norm(a); }
inline V3 P(const double* xyz, int i) { return {xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]}; }
inline void addf(double* f, int i, V3 v) { f[3 * i] += v.x; f[3 * i + 1] += v.y; f[3 * i + 2] += v.z; }
inline void subf(double* f, int i, V3 v) { f[3 * i] -= v.x; f[3 * i + 1] -= v.y; f[3 * i + 2] -= v.z; }

bool no_cutoff(double c) { return !(c > 0.0) || c >= 1e30; }

// Dense exclusion lookup for the oracle's O(n^2) loops: 0, 1 (excluded), 2 (1-4).
std::vector<int8_t> excl_matrix(const og_topology* t) {
  const int n = t->n_atoms;
  std::vector<int8_t> m(static_cast<size_t>(n) * n, 0);
  for (int k = 0; k < t->n_exclusions; ++k) {
    int i = t->exclusion_atoms[2 * k], j = t->exclusion_atoms[2 * k + 1];
    m[static_cast<size_t>(i) * n + j] = t->exclusion_kind[k];
    m[static_cast<size_t>(j) * n + i] = t->exclusion_kind[k];
  }
  return m;
}

// geom/src/measure.rs:9-13
double measure_angle(V3 a, V3 b, V3 c) {
  V3 ba = normalize(a - b), bc = normalize(c - b);
  double x = dot(ba, bc);
  x = x < -1.0 ? -1.0 : (x > 1.0 ? 1.0 : x);
  return std::acos(x);
}

// geom/src/measure.rs:18-28
double measure_dihedral(V3 a, V3 b, V3 c, V3 d) {
  V3 b0 = a - b;
  V3 b1 = normalize(c - b);
  V3 b2 = d - c;
  V3 v = b0 - b1 * dot(b0, b1);
  V3 w = b2 - b1 * dot(b2, b1);
  double x = dot(v, w);
  double y = dot(cross(b1, v), w);
  return std::atan2(y, x);
}

// energy/src/gb.rs:347-369
double pairwise_descreening(double r, double rho_i_tilde, double s_rho_j_tilde) {
  if (r + s_rho_j_tilde <= rho_i_tilde) return 0.0;
  double l = (r - s_rho_j_tilde < rho_i_tilde) ? rho_i_tilde : r - s_rho_j_tilde;
  double u = r + s_rho_j_tilde;
  if (u <= 0.0 || l <= 0.0) return 0.0;
  double inv_l = 1.0 / l, inv_u = 1.0 / u;
  double term1 = 0.5 * (inv_l - inv_u);
  double term2 = (r / 4.0) * (inv_u * inv_u - inv_l * inv_l);
  double term3 = (1.0 / (2.0 * r)) * std::log(l / u);
  double term4 = (s_rho_j_tilde * s_rho_j_tilde - r * r) / (4.0 * r) * (inv_u * inv_u - inv_l * inv_l);
  return term1 + term2 + term3 + term4;
}

// energy/src/forces_bonded.rs:124-167 dihedral_gradient
bool dihedral_gradient(V3 pa, V3 pb, V3 pc, V3 pd, V3* da, V3* db, V3* dc, V3* dd, double* phi) {
  V3 b1 = pb - pa, b2 = pc - pb, b3 = pd - pc;
  double b2n = norm(b2);
  if (b2n < 1e-9) return false;
  V3 s = cross(b1, b2), t = cross(b2, b3);
  double s2 = norm2(s), t2 = norm2(t);
  if (s2 < 1e-18 || t2 < 1e-18) return false;
  *da = s * (b2n / s2);
  *dd = -t * (b2n / t2);
  double inv_b2n_sq = 1.0 / (b2n * b2n);
  double f1 = dot(b1, b2) * inv_b2n_sq;
  double f2 = dot(b3, b2) * inv_b2n_sq;
  *db = (*da) * (-(f1 + 1.0)) + (*dd) * f2;
  *dc = -((*da + *db) + *dd);
  V3 m1 = cross(s, b2 / b2n);
  *phi = std::atan2(dot(m1, t), dot(s, t));
  return true;
}

double wrap_pi(double d) {
  while (d > M_PI) d -= 2.0 * M_PI;
  while (d < -M_PI) d += 2.0 * M_PI;
  return d;
}

// energy/src/forces_bonded.rs:47-236 (add_bond/angle/dihedral/improper_forces)
void bonded_forces(const og_topology* t, const double* xyz, double* f) {
  for (int k = 0; k < t->n_bonds; ++k) {
    int a = t->bond_atoms[2 * k], b = t->bond_atoms[2 * k + 1];
    V3 d = P(xyz, b) - P(xyz, a);
    double r = norm(d);
    if (r < 1e-9) continue;
    double dr = r - t->bond_r0[k];
    double mag = (2.0 * t->bond_k[k] * dr) * kKcalToKj;
    V3 fv = d * (mag / r);
    addf(f, a, fv);
    subf(f, b, fv);
  }
  for (int k = 0; k < t->n_angles; ++k) {
    int a = t->angle_atoms[3 * k], b = t->angle_atoms[3 * k + 1], c = t->angle_atoms[3 * k + 2];
    V3 u = P(xyz, a) - P(xyz, b), v = P(xyz, c) - P(xyz, b);
    double un = norm(u), vn = norm(v);
    if (un < 1e-9 || vn < 1e-9) continue;
    V3 uh = u / un, vh = v / vn;
    double ct = dot(uh, vh);
    ct = ct < -1.0 ? -1.0 : (ct > 1.0 ? 1.0 : ct);
    double st = std::sqrt(1.0 - ct * ct);
    if (st < 1e-9) continue;
    double theta = std::acos(ct);
    double dv = 2.0 * t->angle_k[k] * (theta - deg2rad(t->angle_theta0[k]));
    double coeff = dv * kKcalToKj / st;
    V3 fa = (vh - uh * ct) * (coeff / un);
    V3 fc = (uh - vh * ct) * (coeff / vn);
    V3 fb = -(fa + fc);
    addf(f, a, fa);
    addf(f, b, fb);
    addf(f, c, fc);
  }
  for (int k = 0; k < t->n_dihedrals; ++k) {
    const int* q = t->dihedral_atoms + 4 * k;
    V3 da, db, dc, dd;
    double phi;
    if (!dihedral_gradient(P(xyz, q[0]), P(xyz, q[1]), P(xyz, q[2]), P(xyz, q[3]), &da, &db, &dc, &dd, &phi)) continue;
    double dvdphi = 0.0;
    for (int m = t->dihedral_term_start[k]; m < t->dihedral_term_start[k + 1]; ++m) {
      double arg = t->term_n[m] * phi - deg2rad(t->term_delta[m]);
      dvdphi += -t->term_k[m] * static_cast<double>(t->term_n[m]) * std::sin(arg);
    }
    dvdphi *= kKcalToKj;
    subf(f, q[0], da * dvdphi);
    subf(f, q[1], db * dvdphi);
    subf(f, q[2], dc * dvdphi);
    subf(f, q[3], dd * dvdphi);
  }
  for (int k = 0; k < t->n_impropers; ++k) {
    const int* q = t->improper_atoms + 4 * k;
    V3 da, db, dc, dd;
    double om;
    if (!dihedral_gradient(P(xyz, q[0]), P(xyz, q[1]), P(xyz, q[2]), P(xyz, q[3]), &da, &db, &dc, &dd, &om)) continue;
    double dom = wrap_pi(om - deg2rad(t->improper_psi0[k]));
    double dv = (2.0 * t->improper_k[k] * dom) * kKcalToKj;
    subf(f, q[0], da * dv);
    subf(f, q[1], db * dv);
    subf(f, q[2], dc * dv);
    subf(f, q[3], dd * dv);
  }
}

// Born radii, energy/src/gb.rs:100-144 (compute_born_inputs) and :326-341.
int born_radii(const og_topology* t, const double* xyz, double born_cutoff, double* R) {
  const int n = t->n_atoms;
  std::vector<double> rt(n), integral(n, 0.0);
  for (int i = 0; i < n; ++i) rt[i] = t->gb_rho[i] - kObcOffset;
  const bool all = no_cutoff(born_cutoff);
  const double c2 = born_cutoff * born_cutoff;
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < n; ++i) {
    double acc = 0.0;
    for (int j = 0; j < n; ++j) {
      if (j == i) continue;
      double r2 = norm2(P(xyz, j) - P(xyz, i));
      if ((!all && r2 > c2) || r2 < 1e-18) continue;
      double r = std::sqrt(r2);
      acc += pairwise_descreening(r, rt[i], t->gb_scale[j] * rt[j]);
    }
    integral[i] = acc;
  }
  int clamped = 0;
  for (int i = 0; i < n; ++i) {
    double psi = integral[i] * rt[i];
    double arg = kObcAlpha * psi - kObcBeta * psi * psi + kObcGamma * psi * psi * psi;
    double inv = 1.0 / rt[i] - std::tanh(arg) / t->gb_rho[i];
    double floor_r = rt[i] > 0.5 ? rt[i] : 0.5;
    if (inv <= 0.0 || !std::isfinite(inv)) {
      ++clamped;
      R[i] = floor_r;
    } else {
      double r = 1.0 / inv;
      R[i] = r > floor_r ? r : floor_r;
    }
  }
  return clamped;
}

}  // namespace

extern "C" {

// ---------------------------------------------------------------- energies

// energy/src/bonded.rs:34-191.  out = {bond, angle, dihedral, improper} kJ/mol.
void orc_bonded_energy(const og_topology* t, const double* xyz, double* out) {
  double eb = 0, ea = 0, ed = 0, ei = 0;
  for (int k = 0; k < t->n_bonds; ++k) {
    double r = norm(P(xyz, t->bond_atoms[2 * k + 1]) - P(xyz, t->bond_atoms[2 * k]));
    double dr = r - t->bond_r0[k];
    eb += t->bond_k[k] * dr * dr;
  }
  for (int k = 0; k < t->n_angles; ++k) {
    const int* q = t->angle_atoms + 3 * k;
    double th = measure_angle(P(xyz, q[0]), P(xyz, q[1]), P(xyz, q[2]));
    double d = th - deg2rad(t->angle_theta0[k]);
    ea += t->angle_k[k] * d * d;
  }
  for (int k = 0; k < t->n_dihedrals; ++k) {
    const int* q = t->dihedral_atoms + 4 * k;
    double chi = measure_dihedral(P(xyz, q[0]), P(xyz, q[1]), P(xyz, q[2]), P(xyz, q[3]));
    for (int m = t->dihedral_term_start[k]; m < t->dihedral_term_start[k + 1]; ++m)
      ed += t->term_k[m] * (1.0 + std::cos(t->term_n[m] * chi - deg2rad(t->term_delta[m])));
  }
  for (int k = 0; k < t->n_impropers; ++k) {
    const int* q = t->improper_atoms + 4 * k;
    double om = measure_dihedral(P(xyz, q[0]), P(xyz, q[1]), P(xyz, q[2]), P(xyz, q[3]));
    double d = wrap_pi(om - deg2rad(t->improper_psi0[k]));
    ei += t->improper_k[k] * d * d;
  }
  out[0] = eb * kKcalToKj;
  out[1] = ea * kKcalToKj;
  out[2] = ed * kKcalToKj;
  out[3] = ei * kKcalToKj;
}

// energy/src/nonbonded.rs:97-174.  out = {lj, coulomb} kJ/mol; returns pair count.
int orc_nonbonded_energy(const og_topology* t, const double* xyz, double cutoff, double* out) {
  const int n = t->n_atoms;
  auto ex = excl_matrix(t);
  const bool all = no_cutoff(cutoff);
  const double c2 = cutoff * cutoff;
  const double kappa = all ? 0.0 : 1.0 / (2.0 * cutoff * cutoff * cutoff);
  const double cc = all ? 0.0 : 3.0 / (2.0 * cutoff);
  double lj = 0.0, coul = 0.0;
  long pairs = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : lj, coul, pairs)
  for (int i = 0; i < n; ++i) {
    for (int j = i + 1; j < n; ++j) {
      double r2 = norm2(P(xyz, i) - P(xyz, j));
      if (!all && r2 > c2) continue;
      int8_t m = ex[static_cast<size_t>(i) * n + j];
      if (m == 1) continue;
      double r = std::sqrt(r2);
      double ri, ei, rj, ej;
      if (m == 2) {
        ri = t->rmin_half_14[i]; ei = t->epsilon_14[i]; rj = t->rmin_half_14[j]; ej = t->epsilon_14[j];
      } else {
        ri = t->rmin_half[i]; ei = t->epsilon[i]; rj = t->rmin_half[j]; ej = t->epsilon[j];
      }
      double rmin = ri + rj, eps = std::sqrt(ei * ej);
      double x = rmin / r;
      double r6 = x * x * x * x * x * x;
      lj += eps * (r6 * r6 - 2.0 * r6);
      double qq = t->charge[i] * t->charge[j];
      if (qq != 0.0) coul += kCoulomb * qq * (1.0 / r + kappa * r * r - cc);
      ++pairs;
    }
  }
  out[0] = lj * kKcalToKj;
  out[1] = coul * kKcalToKj;
  return static_cast<int>(pairs);
}

// Descreening integrals I_i (energy/src/gb.rs:268-324), before the OBC map.
void orc_born_integrals(const og_topology* t, const double* xyz, double born_cutoff, double* out) {
  const int n = t->n_atoms;
  const bool all = no_cutoff(born_cutoff);
  const double c2 = born_cutoff * born_cutoff;
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < n; ++i) {
    double acc = 0.0;
    const double rti = t->gb_rho[i] - kObcOffset;
    for (int j = 0; j < n; ++j) {
      if (j == i) continue;
      double r2 = norm2(P(xyz, j) - P(xyz, i));
      if ((!all && r2 > c2) || r2 < 1e-18) continue;
      acc += pairwise_descreening(std::sqrt(r2), rti, t->gb_scale[j] * (t->gb_rho[j] - kObcOffset));
    }
    out[i] = acc;
  }
}

// energy/src/gb.rs:100-144.  Returns the clamp count.
int orc_born_radii(const og_topology* t, const double* xyz, double born_cutoff, double* radii) {
  return born_radii(t, xyz, born_cutoff, radii);
}

// energy/src/gb.rs:146-182.  out = {gb, self, pair}; pair sum over ALL pairs.
int orc_gb_energy(const og_topology* t, const double* xyz, double born_cutoff, double* out) {
  const int n = t->n_atoms;
  std::vector<double> R(n);
  int clamped = born_radii(t, xyz, born_cutoff, R.data());
  const double pref = -0.5 * (1.0 / 1.0 - 1.0 / kEpsWater) * kCoulomb;
  double self_e = 0.0;
  for (int i = 0; i < n; ++i)
    if (t->charge[i] != 0.0) self_e += pref * (t->charge[i] * t->charge[i]) / R[i];
  double pair_e = 0.0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : pair_e)
  for (int i = 0; i < n; ++i)
    for (int j = i + 1; j < n; ++j) {
      double qq = t->charge[i] * t->charge[j];
      if (qq == 0.0) continue;
      double r2 = norm2(P(xyz, i) - P(xyz, j));
      double rp = R[i] * R[j];
      double fgb = std::sqrt(r2 + rp * std::exp(-r2 / (4.0 * rp)));
      pair_e += 2.0 * pref * qq / fgb;
    }
  out[0] = (self_e + pair_e) * kKcalToKj;
  out[1] = self_e * kKcalToKj;
  out[2] = pair_e * kKcalToKj;
  return clamped;
}

// ------------------------------------------------------------------ forces

// energy/src/forces.rs:78-128 total_force_with_scratch without SASA:
// bonded (forces_bonded.rs) + LJ/RF-Coulomb SoA pair force
// (forces_nonbonded.rs:196-232) + GB frozen-radii pair force with Born radii
// from the descreening pass (forces_gb.rs:51-150).  f is overwritten.
void orc_total_force(const og_topology* t, const double* xyz, double nb_cutoff, double born_cutoff,
                     double gb_cutoff, double* f) {
  const int n = t->n_atoms;
  std::memset(f, 0, sizeof(double) * 3 * n);
  bonded_forces(t, xyz, f);

  auto ex = excl_matrix(t);
  std::vector<double> R(n);
  born_radii(t, xyz, born_cutoff, R.data());
  const bool nb_all = no_cutoff(nb_cutoff), gb_all = no_cutoff(gb_cutoff);
  const double nb_c2 = nb_cutoff * nb_cutoff, gb_c2 = gb_cutoff * gb_cutoff;
  const double inv_rc3 = nb_all ? 0.0 : 1.0 / (nb_cutoff * nb_cutoff * nb_cutoff);
  const double coulomb_kj = kCoulomb * kKcalToKj;
  const double gb_pref = (1.0 / 1.0 - 1.0 / kEpsWater) * kCoulomb * kKcalToKj;

  // Per-atom pair accumulation over j != i (each unordered pair contributes
  // +F to i and -F to j, so summing i's row over every j gives the same total).
  std::vector<double> nbf(3 * n, 0.0);
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < n; ++i) {
    double fx = 0, fy = 0, fz = 0;
    for (int j = 0; j < n; ++j) {
      if (j == i) continue;
      double dx = xyz[3 * j] - xyz[3 * i], dy = xyz[3 * j + 1] - xyz[3 * i + 1], dz = xyz[3 * j + 2] - xyz[3 * i + 2];
      double r2 = dx * dx + dy * dy + dz * dz;
      if (r2 < 1e-18) continue;
      double coeff = 0.0;
      // LJ + reaction-field Coulomb
      int8_t m = ex[static_cast<size_t>(i) * n + j];
      if (m != 1 && (nb_all || r2 <= nb_c2)) {
        double ri, ei, rj, ej;
        if (m == 2) {
          ri = t->rmin_half_14[i]; ei = t->epsilon_14[i]; rj = t->rmin_half_14[j]; ej = t->epsilon_14[j];
        } else {
          ri = t->rmin_half[i]; ei = t->epsilon[i]; rj = t->rmin_half[j]; ej = t->epsilon[j];
        }
        double rmin = ri + rj, eps = std::sqrt(ei * ej);
        double inv_r2 = 1.0 / r2;
        double ratio2 = rmin * rmin * inv_r2;
        double ratio6 = ratio2 * ratio2 * ratio2;
        double ratio12 = ratio6 * ratio6;
        coeff += 12.0 * eps * inv_r2 * (ratio6 - ratio12) * kKcalToKj;
        double qq = t->charge[i] * t->charge[j];
        if (qq != 0.0) coeff += -coulomb_kj * qq * (inv_r2 / std::sqrt(r2) - inv_rc3);
      }
      // GB frozen-radii pair force
      double qq = t->charge[i] * t->charge[j];
      if (qq != 0.0 && (gb_all || r2 <= gb_c2)) {
        double r = std::sqrt(r2);
        double rp = R[i] * R[j];
        double e = std::exp(-r2 / (4.0 * rp));
        double f2 = r2 + rp * e;
        double fgb = std::sqrt(f2);
        double dfdr = (2.0 * r - 0.5 * r * e) / (2.0 * fgb);
        coeff += gb_pref * qq / f2 * dfdr / r;
      }
      fx += dx * coeff;
      fy += dy * coeff;
      fz += dz * coeff;
    }
    nbf[3 * i] = fx;
    nbf[3 * i + 1] = fy;
    nbf[3 * i + 2] = fz;
  }
  for (int k = 0; k < 3 * n; ++k) f[k] += nbf[k];
}

// Bonded-only forces (for per-term parity checks).
void orc_bonded_forces(const og_topology* t, const double* xyz, double* f) {
  std::memset(f, 0, sizeof(double) * 3 * t->n_atoms);
  bonded_forces(t, xyz, f);
}

// Potential energy as origami's REMD swap / L-BFGS line search compute it
// (dynamics/src/remd.rs:529-539, energy_eval.rs:20-34), without SASA.
// terms (optional, 9 doubles): bond angle dihedral improper lj coulomb gb gb_self gb_pair.
double orc_potential_energy(const og_topology* t, const double* xyz, double nb_cutoff, double born_cutoff,
                            double* terms) {
  double b[4], nb[2], gb[3];
  orc_bonded_energy(t, xyz, b);
  orc_nonbonded_energy(t, xyz, nb_cutoff, nb);
  orc_gb_energy(t, xyz, born_cutoff, gb);
  if (terms) {
    for (int k = 0; k < 4; ++k) terms[k] = b[k];
    terms[4] = nb[0]; terms[5] = nb[1];
    terms[6] = gb[0]; terms[7] = gb[1]; terms[8] = gb[2];
  }
  return b[0] + b[1] + b[2] + b[3] + nb[0] + nb[1] + gb[0];
}

// Exclusion classification straight from the TopologyGraph predicates
// (geom/src/topology_graph.rs:81-112, energy/src/scratch.rs:233-251): O(n^2)
// over the bond list; out is n*n bytes (0, 1 excluded, 2 = 1-4).
void orc_exclusion_matrix(int n, int n_bonds, const int32_t* bonds, int8_t* out) {
  std::vector<std::vector<int>> adj(n);
  for (int k = 0; k < n_bonds; ++k) {
    adj[bonds[2 * k]].push_back(bonds[2 * k + 1]);
    adj[bonds[2 * k + 1]].push_back(bonds[2 * k]);
  }
  auto has = [&](int a, int b) {
    for (int x : adj[a]) if (x == b) return true;
    return false;
  };
  auto bonded = [&](int a, int b) { return has(a, b); };
  auto one_three = [&](int a, int b) {
    if (a == b) return false;
    for (int m : adj[a]) if (has(m, b)) return true;
    return false;
  };
  auto one_four = [&](int a, int b) {
    if (a == b || bonded(a, b) || one_three(a, b)) return false;
    for (int n1 : adj[a]) for (int n2 : adj[n1]) if (has(n2, b)) return true;
    return false;
  };
  std::memset(out, 0, static_cast<size_t>(n) * n);
  for (int i = 0; i < n; ++i)
    for (int j = i + 1; j < n; ++j) {
      int8_t m = (bonded(i, j) || one_three(i, j)) ? 1 : (one_four(i, j) ? 2 : 0);
      out[static_cast<size_t>(i) * n + j] = m;
      out[static_cast<size_t>(j) * n + i] = m;
    }
}

// ------------------------------------------------------------------ random

// xoshiro256++ seeded by SplitMix64, Box-Muller with a cached spare
// (dynamics/src/rng.rs:18-98).
struct orc_xoshiro {
  uint64_t s[4];
  int has_spare;
  double spare;
};

static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

void orc_xoshiro_seed(orc_xoshiro* r, uint64_t seed) {
  uint64_t sm = seed;
  for (int k = 0; k < 4; ++k) {
    sm += 0x9e3779b97f4a7c15ULL;
    uint64_t z = sm;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    r->s[k] = z ^ (z >> 31);
  }
  r->has_spare = 0;
  r->spare = 0.0;
}

uint64_t orc_xoshiro_u64(orc_xoshiro* r) {
  uint64_t* s = r->s;
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

double orc_xoshiro_f64(orc_xoshiro* r) {
  return static_cast<double>(orc_xoshiro_u64(r) >> 11) * (1.0 / static_cast<double>(1ULL << 53));
}

double orc_xoshiro_gaussian(orc_xoshiro* r) {
  if (r->has_spare) {
    r->has_spare = 0;
    return r->spare;
  }
  double u1 = orc_xoshiro_f64(r);
  while (u1 <= 0.0) u1 = orc_xoshiro_f64(r);
  double u2 = orc_xoshiro_f64(r);
  double rr = std::sqrt(-2.0 * std::log(u1));
  double th = 2.0 * M_PI * u2;
  r->spare = rr * std::sin(th);
  r->has_spare = 1;
  return rr * std::cos(th);
}

int orc_xoshiro_size(void) { return static_cast<int>(sizeof(orc_xoshiro)); }

// ------------------------------------------------------- engine noise model
// The GPU engine's O-step noise: Philox4x32-10 with counter (atom, step_lo,
// step_hi, system) and key (seed_lo, seed_hi); two Box-Muller pairs give the
// x, y (pair 1) and z (pair 2, cosine) normals.  Restated here so integrator
// trajectories can be compared step for step.
void orc_engine_normals(uint64_t seed, uint32_t sys, uint64_t step, uint32_t atom, double* out3) {
  uint32_t c0 = atom, c1 = static_cast<uint32_t>(step), c2 = static_cast<uint32_t>(step >> 32), c3 = sys;
  uint32_t k0 = static_cast<uint32_t>(seed), k1 = static_cast<uint32_t>(seed >> 32);
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = static_cast<uint64_t>(0xD2511F53u) * c0;
    uint64_t p1 = static_cast<uint64_t>(0xCD9E8D57u) * c2;
    uint32_t hi0 = static_cast<uint32_t>(p0 >> 32), lo0 = static_cast<uint32_t>(p0);
    uint32_t hi1 = static_cast<uint32_t>(p1 >> 32), lo1 = static_cast<uint32_t>(p1);
    uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  auto open01 = [](uint32_t v) { return (static_cast<double>(v) + 1.0) * (1.0 / 4294967296.0); };
  double m1 = std::sqrt(-2.0 * std::log(open01(c0)));
  double m2 = std::sqrt(-2.0 * std::log(open01(c2)));
  double a1 = 2.0 * M_PI * (static_cast<double>(c1) * (1.0 / 4294967296.0));
  double a2 = 2.0 * M_PI * (static_cast<double>(c3) * (1.0 / 4294967296.0));
  out3[0] = m1 * std::cos(a1);
  out3[1] = m1 * std::sin(a1);
  out3[2] = m2 * std::cos(a2);
}

// dynamics/src/shake.rs:86-125 (global Gauss-Seidel passes).  Returns the
// pass count, or -1 when not converged.
int orc_shake(double* pos, const double* ref, const double* inv_mass, int n_cons, const int32_t* cons,
              const double* d, double tol_sq, int max_iters) {
  for (int iter = 1; iter <= max_iters; ++iter) {
    double max_err = 0.0;
    for (int c = 0; c < n_cons; ++c) {
      int i = cons[2 * c], j = cons[2 * c + 1];
      V3 rn = P(pos, i) - P(pos, j);
      double err = norm2(rn) - d[c] * d[c];
      if (std::fabs(err) > max_err) max_err = std::fabs(err);
      if (std::fabs(err) < tol_sq) continue;
      V3 ro = P(ref, i) - P(ref, j);
      double denom = 2.0 * (inv_mass[i] + inv_mass[j]) * dot(rn, ro);
      if (std::fabs(denom) < 1e-18) continue;
      V3 delta = ro * (err / denom);
      subf(pos, i, delta * inv_mass[i]);
      addf(pos, j, delta * inv_mass[j]);
    }
    if (max_err < tol_sq) return iter;
  }
  return -1;
}

// The BAOAB(+SHAKE) loop body of dynamics/src/langevin.rs:223-313 with the
// engine's noise model, for n_steps starting at step index step0 + 1.
// xyz, v, f are updated in place (f must hold the forces at xyz on entry).
// Returns the number of SHAKE half-steps that failed to converge.
int orc_baoab(const og_topology* t, double* xyz, double* v, double* f, int n_steps, double dt, double gamma_ps,
              double temperature, int use_shake, uint64_t seed, uint32_t sys, uint64_t step0, double nb_cutoff,
              double born_cutoff, double gb_cutoff) {
  const int n = t->n_atoms;
  const double alpha = std::exp(-gamma_ps * dt * 1.0e-3);
  const double kbt = kBoltzmann * temperature;
  const double h = 0.5 * dt;
  std::vector<double> inv_m(n), ref(3 * n);
  for (int i = 0; i < n; ++i) inv_m[i] = 1.0 / t->mass[i];
  const bool shake = use_shake && t->n_constraints > 0;
  const double dof = 3.0 * n;
  const double dof_corr = shake ? dof / std::max(dof - t->n_constraints, 1.0) : 1.0;
  int failures = 0;
  auto b_step = [&]() {
    for (int i = 0; i < n; ++i) {
      double c = (kAccel / t->mass[i]) * h;
      for (int k = 0; k < 3; ++k) v[3 * i + k] += f[3 * i + k] * c;
    }
  };
  auto a_step = [&]() {
    if (shake) std::memcpy(ref.data(), xyz, sizeof(double) * 3 * n);
    for (int k = 0; k < 3 * n; ++k) xyz[k] += v[k] * h;
    if (shake) {
      if (orc_shake(xyz, ref.data(), inv_m.data(), t->n_constraints, t->constraint_atoms, t->constraint_length,
                    1e-6, 64) < 0)
        ++failures;
      for (int k = 0; k < 3 * n; ++k) v[k] = (xyz[k] - ref[k]) / h;
    }
  };
  for (int s = 1; s <= n_steps; ++s) {
    const uint64_t step = step0 + static_cast<uint64_t>(s);
    b_step();
    a_step();
    const double oma2 = 1.0 - alpha * alpha;
    for (int i = 0; i < n; ++i) {
      double sigma = std::sqrt(oma2 * kbt * dof_corr * kAccel / t->mass[i]);
      double xi[3];
      orc_engine_normals(seed, sys, step, static_cast<uint32_t>(i), xi);
      for (int k = 0; k < 3; ++k) v[3 * i + k] = alpha * v[3 * i + k] + sigma * xi[k];
    }
    a_step();
    orc_total_force(t, xyz, nb_cutoff, born_cutoff, gb_cutoff, f);
    b_step();
  }
  return failures;
}

}  // extern "C"
