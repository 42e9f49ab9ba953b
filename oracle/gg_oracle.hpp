// gg_oracle.hpp -- CPU oracle for the gargantua GR ray path.
//
// TEST INFRASTRUCTURE ONLY.  This header restates, in plain C++17 double
// arithmetic, the reference's f64 CPU path (gargantua, a Rust workspace).  It
// is the checker the CUDA kernels are compared with and the timed CPU
// baseline; nothing in the product links it.  Only tests/, the smoke check
// and the CPU-baseline leg of bench.py load it.
//
// Pinning: the reference cannot be built here (Rust, no toolchain, crates not
// vendored), and its tests hold no golden vectors for RK45 endpoints or
// images.  This restatement is pinned against every known-answer test the
// reference's own tests hold for the path (metric values, horizon, analytic
// vs numerical Christoffels, circular orbits, Keplerian normalisation, the
// 32x24 render sanity check) and against an independent pure-Python
// restatement (tests/golden/make_golden.py) on seeded rays.  RK45 endpoint
// parity is otherwise unpinned by the reference itself.
//
// Operation order follows the Rust source expression by expression (Rust
// never contracts a*b+c into an FMA, so this file is built with
// -ffp-contract=off).  Each function cites the reference file:line it follows.
// Items marked EXTENSION are new specifications (thin disk, checkerboard
// sky, rtol/atol error norm, jitter, inclined camera, ISCO / photon orbit)
// that do not exist in the reference; they sit on top of the exact core.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace ggo {

constexpr double kPi = 3.14159265358979323846;

// ---------------------------------------------------------------------------
// Small vector types standing in for nalgebra Vector3/Vector4.
// nalgebra's norm() is sqrt of a left-to-right sum of squares for these
// sizes; normalize() divides each component by the norm.
// ---------------------------------------------------------------------------
template <class T>
struct V4 {
  T c[4];
  T& operator[](int i) { return c[i]; }
  const T& operator[](int i) const { return c[i]; }
};
template <class T>
inline V4<T> operator+(const V4<T>& a, const V4<T>& b) {
  return {{a[0] + b[0], a[1] + b[1], a[2] + b[2], a[3] + b[3]}};
}
template <class T>
inline V4<T> operator-(const V4<T>& a, const V4<T>& b) {
  return {{a[0] - b[0], a[1] - b[1], a[2] - b[2], a[3] - b[3]}};
}
template <class T>
inline V4<T> operator*(const T& s, const V4<T>& v) {
  return {{s * v[0], s * v[1], s * v[2], s * v[3]}};
}
template <class T>
inline T norm(const V4<T>& v) {
  using std::sqrt;
  T s = v[0] * v[0];
  s = s + v[1] * v[1];
  s = s + v[2] * v[2];
  s = s + v[3] * v[3];
  return sqrt(s);
}

struct V3 {
  double c[3];
  double& operator[](int i) { return c[i]; }
  const double& operator[](int i) const { return c[i]; }
};
inline V3 operator+(const V3& a, const V3& b) { return {{a[0] + b[0], a[1] + b[1], a[2] + b[2]}}; }
inline V3 operator*(double s, const V3& v) { return {{s * v[0], s * v[1], s * v[2]}}; }
inline double dot(const V3& a, const V3& b) {
  double s = a[0] * b[0];
  s = s + a[1] * b[1];
  s = s + a[2] * b[2];
  return s;
}
inline double norm(const V3& v) { return std::sqrt(dot(v, v)); }
inline V3 normalize(const V3& v) {
  double n = norm(v);
  return {{v[0] / n, v[1] / n, v[2] / n}};
}
inline V3 cross(const V3& a, const V3& b) {
  return {{a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]}};
}

// f64::max / clamp / rem_euclid semantics (NaN-ignoring max like Rust).
template <class T>
inline T rmax(const T& a, const T& b) {
  using std::fmax;
  return fmax(a, b);
}
template <class T>
inline T rclamp(const T& x, double lo, double hi) {
  if (x < T(lo)) return T(lo);
  if (x > T(hi)) return T(hi);
  return x;
}
template <class T>
inline T rem_euclid(const T& x, double m) {
  using std::fmod;
  T r = fmod(x, T(m));
  if (r < T(0.0)) return r + T(m);
  return r;
}

// ---------------------------------------------------------------------------
// Metric tensor as the five independent Boyer-Lindquist components.
// ---------------------------------------------------------------------------
template <class T>
struct G {
  T tt, rr, thth, phph, tph;
};

// Schwarzschild (crates/gr-core/src/schwarzschild.rs)
struct Schwarzschild {
  double mass, rs;
  explicit Schwarzschild(double m) : mass(m), rs(2.0 * m) {}  // :13-18

  template <class T>
  G<T> metric_tensor(const V4<T>& pos) const {  // :26-43
    using std::sin;
    T r = pos[1];
    T theta = pos[2];
    r = rmax(r, T(1e-10));
    T f = T(1.0) - T(rs) / r;
    T sin_theta = sin(theta);
    G<T> g;
    g.tt = -f;
    g.rr = T(1.0) / f;
    g.thth = r * r;
    g.phph = r * r * sin_theta * sin_theta;
    g.tph = T(0.0);
    return g;
  }

  template <class T>
  void christoffel(const V4<T>& pos, T gamma[4][4][4]) const {  // :45-88
    using std::cos;
    using std::sin;
    T r = rmax(pos[1], T(1e-10));
    T theta = pos[2];
    T sin_theta = sin(theta);
    T cos_theta = cos(theta);
    T rsT(rs);
    for (int i = 0; i < 64; ++i) (&gamma[0][0][0])[i] = T(0.0);
    gamma[0][0][1] = rsT / (T(2.0) * r * (r - rsT));
    gamma[0][1][0] = gamma[0][0][1];
    gamma[1][0][0] = rsT * (r - rsT) / (T(2.0) * r * r * r);
    gamma[1][1][1] = -rsT / (T(2.0) * r * (r - rsT));
    gamma[1][2][2] = -(r - rsT);
    gamma[1][3][3] = -(r - rsT) * sin_theta * sin_theta;
    gamma[2][1][2] = T(1.0) / r;
    gamma[2][2][1] = T(1.0) / r;
    gamma[2][3][3] = -sin_theta * cos_theta;
    gamma[3][1][3] = T(1.0) / r;
    gamma[3][3][1] = T(1.0) / r;
    gamma[3][2][3] = cos_theta / sin_theta;
    gamma[3][3][2] = gamma[3][2][3];
  }

  // Inlined sparse RHS (:99-140).
  template <class T>
  V4<T> geodesic_acceleration(const V4<T>& pos, const V4<T>& vel) const {
    using std::cos;
    using std::sin;
    T r = rmax(pos[1], T(1e-10));
    T theta = pos[2];
    T sin_theta = sin(theta);
    T cos_theta = cos(theta);
    T rsT(rs);
    T f_denom = r * (r - rsT);
    T rmrs = r - rsT;
    T inv_r = T(1.0) / r;
    T g_t_tr = rsT / (T(2.0) * f_denom);
    T g_r_tt = rsT * rmrs / (T(2.0) * r * r * r);
    T g_r_rr = -rsT / (T(2.0) * f_denom);
    T g_r_thth = -rmrs;
    T g_r_phph = -rmrs * sin_theta * sin_theta;
    T g_th_phph = -sin_theta * cos_theta;
    T g_ph_thph = cos_theta / sin_theta;
    T vt = vel[0], vr = vel[1], vth = vel[2], vph = vel[3];
    T acc_t = T(-2.0) * g_t_tr * vt * vr;
    T acc_r = -g_r_tt * vt * vt - g_r_rr * vr * vr - g_r_thth * vth * vth - g_r_phph * vph * vph;
    T acc_th = T(-2.0) * inv_r * vr * vth - g_th_phph * vph * vph;
    T acc_ph = T(-2.0) * inv_r * vr * vph - T(2.0) * g_ph_thph * vth * vph;
    return {{acc_t, acc_r, acc_th, acc_ph}};
  }

  bool event_horizon(double* rh) const {  // :142-144
    *rh = rs;
    return true;
  }

  // :146-153
  template <class T>
  bool orbital_four_velocity(const V4<T>& pos, V4<T>* u) const;
};

// Kerr in Boyer-Lindquist coordinates (crates/gr-core/src/kerr.rs)
struct Kerr {
  double mass, spin;
  // Kerr::new (:29-34); the assert on mass > 0 is the caller's job here.
  Kerr(double m, double a) : mass(m) {
    double max_spin = m * 0.9999;
    spin = a < -max_spin ? -max_spin : (a > max_spin ? max_spin : a);
  }

  template <class T>
  T sigma(const T& r, const T& theta) const {  // :38-42
    using std::cos;
    T a(spin);
    T cos_theta = cos(theta);
    return r * r + a * a * cos_theta * cos_theta;
  }
  template <class T>
  T delta(const T& r) const {  // :46-50
    T m(mass), a(spin);
    return r * r - T(2.0) * m * r + a * a;
  }

  template <class T>
  G<T> metric_tensor(const V4<T>& pos) const {  // :61-94
    using std::sin;
    T r = rmax(pos[1], T(1e-10));
    T theta = pos[2];
    T m(mass), a(spin);
    T a2 = a * a;
    T sig = sigma(r, theta);
    T del = delta(r);
    T sin_theta = sin(theta);
    T sin2 = sin_theta * sin_theta;
    G<T> g;
    g.tt = -(T(1.0) - T(2.0) * m * r / sig);
    g.rr = sig / del;
    g.thth = sig;
    g.phph = (r * r + a2 + T(2.0) * m * a2 * r * sin2 / sig) * sin2;
    g.tph = T(-2.0) * m * a * r * sin2 / sig;
    return g;
  }

  // Analytic Christoffels (:100-424), expression by expression.
  template <class T>
  void christoffel(const V4<T>& pos, T gamma[4][4][4]) const {
    using std::cos;
    using std::sin;
    T r = rmax(pos[1], T(1e-10));
    T theta = pos[2];
    T m(mass), a(spin);
    T a2 = a * a;
    T sig = sigma(r, theta);
    T del = delta(r);
    T sin_theta = sin(theta);
    T cos_theta = cos(theta);
    T sin2 = sin_theta * sin_theta;
    T sigma2 = sig * sig;
    T r2 = r * r;
    T dsigma_dr = T(2.0) * r;
    T dsigma_dtheta = T(-2.0) * a2 * sin_theta * cos_theta;
    T ddelta_dr = T(2.0) * r - T(2.0) * m;
    T r2_plus_a2 = r2 + a2;
    T big_a = r2_plus_a2 * r2_plus_a2 - a2 * del * sin2;
    T g_inv_tt = -big_a / (sig * del);
    T g_inv_tphi = T(-2.0) * m * a * r / (sig * del);
    T g_inv_rr = del / sig;
    T g_inv_thth = T(1.0) / sig;
    T g_inv_phph = (del - a2 * sin2) / (sig * del * sin2);
    T dg_tt_dr = T(2.0) * m / sig - T(2.0) * m * r * dsigma_dr / sigma2;
    T dg_tt_dth = T(-2.0) * m * r * dsigma_dtheta / sigma2;
    T dg_rr_dr = (dsigma_dr * del - sig * ddelta_dr) / (del * del);
    T dg_rr_dth = dsigma_dtheta / del;
    T dg_thth_dr = dsigma_dr;
    T dg_thth_dth = dsigma_dtheta;
    T big_p = T(2.0) * m * a2 * r;
    // The reference also computes an unused first form of dg_phph_dr
    // (:180-181) and overrides it with this one (:187-188, :208).
    T dg_phph_dr =
        T(2.0) * r * sin2 + sin2 * sin2 * T(2.0) * m * a2 * (sig - T(2.0) * r2) / sigma2;
    T dg_phph_dth = T(2.0) * r2_plus_a2 * sin_theta * cos_theta +
                    big_p *
                        (T(4.0) * sin_theta * sin_theta * sin_theta * cos_theta * sig -
                         sin2 * sin2 * dsigma_dtheta) /
                        sigma2;
    T dg_tphi_dr = T(-2.0) * m * a * sin2 * (sig - r * dsigma_dr) / sigma2;
    T dg_tphi_dth =
        T(-2.0) * m * a * r * (T(2.0) * sin_theta * cos_theta * sig - sin2 * dsigma_dtheta) /
        sigma2;

    for (int i = 0; i < 64; ++i) (&gamma[0][0][0])[i] = T(0.0);
    T val;
    val = T(0.5) * (g_inv_tt * dg_tt_dr + g_inv_tphi * dg_tphi_dr);
    gamma[0][0][1] = val; gamma[0][1][0] = val;
    val = T(0.5) * (g_inv_tt * dg_tt_dth + g_inv_tphi * dg_tphi_dth);
    gamma[0][0][2] = val; gamma[0][2][0] = val;
    val = T(0.5) * (g_inv_tt * dg_tphi_dr + g_inv_tphi * dg_phph_dr);
    gamma[0][1][3] = val; gamma[0][3][1] = val;
    val = T(0.5) * (g_inv_tt * dg_tphi_dth + g_inv_tphi * dg_phph_dth);
    gamma[0][2][3] = val; gamma[0][3][2] = val;

    gamma[1][0][0] = T(-0.5) * g_inv_rr * dg_tt_dr;
    gamma[1][1][1] = T(0.5) * g_inv_rr * dg_rr_dr;
    gamma[1][2][2] = T(-0.5) * g_inv_rr * dg_thth_dr;
    gamma[1][3][3] = T(-0.5) * g_inv_rr * dg_phph_dr;
    val = T(0.5) * g_inv_rr * dg_rr_dth;
    gamma[1][1][2] = val; gamma[1][2][1] = val;
    val = T(-0.5) * g_inv_rr * dg_tphi_dr;
    gamma[1][0][3] = val; gamma[1][3][0] = val;

    gamma[2][0][0] = T(-0.5) * g_inv_thth * dg_tt_dth;
    gamma[2][1][1] = T(-0.5) * g_inv_thth * dg_rr_dth;
    gamma[2][2][2] = T(0.5) * g_inv_thth * dg_thth_dth;
    gamma[2][3][3] = T(-0.5) * g_inv_thth * dg_phph_dth;
    val = T(0.5) * g_inv_thth * dg_thth_dr;
    gamma[2][1][2] = val; gamma[2][2][1] = val;
    val = T(-0.5) * g_inv_thth * dg_tphi_dth;
    gamma[2][0][3] = val; gamma[2][3][0] = val;

    val = T(0.5) * (g_inv_tphi * dg_tt_dr + g_inv_phph * dg_tphi_dr);
    gamma[3][0][1] = val; gamma[3][1][0] = val;
    val = T(0.5) * (g_inv_tphi * dg_tt_dth + g_inv_phph * dg_tphi_dth);
    gamma[3][0][2] = val; gamma[3][2][0] = val;
    val = T(0.5) * (g_inv_tphi * dg_tphi_dr + g_inv_phph * dg_phph_dr);
    gamma[3][1][3] = val; gamma[3][3][1] = val;
    val = T(0.5) * (g_inv_tphi * dg_tphi_dth + g_inv_phph * dg_phph_dth);
    gamma[3][2][3] = val; gamma[3][3][2] = val;
    gamma[3][0][0] = T(0.0);
  }

  // Kerr has no RHS override: the trait default (crates/gr-core/src/metric.rs:37-52)
  // contracts the dense Christoffel array in mu, alpha, beta order.
  template <class T>
  V4<T> geodesic_acceleration(const V4<T>& pos, const V4<T>& vel) const {
#ifdef GGO_ALT_KERR_RHS
    // NOT the reference formulation.  Built only into liboracle_gg_alt.so,
    // whose deviation from the plain build measures how much each ray's
    // endpoint moves when the same right-hand side is rounded through a
    // different (algebraically equivalent) arrangement: the 20 non-zero
    // symbols folded into the contraction, one reciprocal for 1/Sigma,
    // 1/Delta, 1/sin^2.
    return alt_acceleration(pos, vel);
#endif
    T gamma[4][4][4];
    christoffel(pos, gamma);
    V4<T> acc{{T(0.0), T(0.0), T(0.0), T(0.0)}};
    for (int mu = 0; mu < 4; ++mu)
      for (int alpha = 0; alpha < 4; ++alpha)
        for (int beta = 0; beta < 4; ++beta)
          acc[mu] = acc[mu] - gamma[mu][alpha][beta] * vel[alpha] * vel[beta];
    return acc;
  }

  template <class T>
  V4<T> alt_acceleration(const V4<T>& pos, const V4<T>& vel) const {
    using std::cos;
    using std::sin;
    const T r = rmax(pos[1], T(1e-10));
    const T s = sin(pos[2]), c = cos(pos[2]);
    const T M(mass), a(spin);
    const T r2 = r * r, a2 = a * a, s2 = s * s, c2 = c * c, sc = s * c;
    const T sig = r2 + a2 * c2, del = (r - T(2) * M) * r + a2, rho = r2 + a2, sd = sig * del;
    const T R = T(1) / (sd * s2);
    const T iSD = s2 * R, iS = del * iSD, iD = sig * iSD, is2 = sd * R, iS2 = iS * iS;
    const T Mr = M * r, sm2r = a2 * c2 - r2;
    const T dtt_r = T(2) * M * sm2r * iS2, dtt_th = T(4) * Mr * a2 * sc * iS2;
    const T drr_r = T(2) * (a2 * (r * s2 + M * c2) - M * r2) * (iD * iD);
    const T drr_th = T(-2) * a2 * sc * iD;
    const T dthth_r = T(2) * r, dthth_th = T(-2) * a2 * sc;
    const T dphph_r = T(2) * r * s2 + T(2) * M * a2 * (s2 * s2) * sm2r * iS2;
    const T dphph_th = T(2) * rho * sc + T(4) * Mr * a2 * sc * s2 * (sig + rho) * iS2;
    const T dtph_r = T(-2) * M * a * s2 * sm2r * iS2, dtph_th = T(-4) * Mr * a * sc * rho * iS2;
    const T gtt = -(rho * rho - a2 * del * s2) * iSD, gtph = T(-2) * Mr * a * iSD;
    const T gphph = (del - a2 * s2) * iSD * is2;
    const T vt = vel[0], vr = vel[1], vth = vel[2], vph = vel[3];
    const T Et = vr * (dtt_r * vt + dtph_r * vph) + vth * (dtt_th * vt + dtph_th * vph);
    const T Ep = vr * (dtph_r * vt + dphph_r * vph) + vth * (dtph_th * vt + dphph_th * vph);
    const T two_tp = T(2) * vt * vph, two_rt = T(2) * vr * vth;
    V4<T> out;
    out[0] = -(gtt * Et + gtph * Ep);
    out[3] = -(gtph * Et + gphph * Ep);
    out[1] = T(-0.5) * del * iS *
             (drr_r * vr * vr - dtt_r * vt * vt - dthth_r * vth * vth - dphph_r * vph * vph +
              drr_th * two_rt - dtph_r * two_tp);
    out[2] = T(-0.5) * iS *
             (dthth_th * vth * vth - dtt_th * vt * vt - drr_th * vr * vr - dphph_th * vph * vph +
              dthth_r * two_rt - dtph_th * two_tp);
    return out;
  }

  bool event_horizon(double* rh) const {  // :427-436
    double m = mass, a = spin;
    double discriminant = m * m - a * a;
    if (discriminant < 0.0) return false;
    *rh = m + std::sqrt(discriminant);
    return true;
  }

  template <class T>
  bool orbital_four_velocity(const V4<T>& pos, V4<T>* u) const;  // :439-449
};

// circular_orbit_velocity (crates/gr-core/src/metric.rs:82-94)
template <class M, class T>
bool circular_orbit_velocity(const M& metric, const V4<T>& pos, const T& omega, V4<T>* u) {
  using std::isfinite;
  using std::sqrt;
  G<T> g = metric.metric_tensor(pos);
  T denom = -(g.tt + T(2.0) * g.tph * omega + g.phph * omega * omega);
  if (denom <= T(0.0) || !isfinite(denom)) return false;
  T u_t = T(1.0) / sqrt(denom);
  *u = {{u_t, T(0.0), T(0.0), omega * u_t}};
  return true;
}

template <class T>
bool Schwarzschild::orbital_four_velocity(const V4<T>& pos, V4<T>* u) const {
  using std::sqrt;
  T r = pos[1];
  if (r <= T(3.0 * mass)) return false;
  T omega = sqrt(T(mass) / (r * r * r));
  return circular_orbit_velocity(*this, pos, omega, u);
}

template <class T>
bool Kerr::orbital_four_velocity(const V4<T>& pos, V4<T>* u) const {
  using std::pow;
  using std::sqrt;
  T r = pos[1];
  T m(mass), a(spin);
  if (r <= T(0.0)) return false;
  T sqrt_m = sqrt(m);
  T omega = sqrt_m / (pow(r, T(1.5)) + a * sqrt_m);
  return circular_orbit_velocity(*this, pos, omega, u);
}

// Numerical Christoffels by central differences (metric.rs:97-142 and the
// test helper kerr.rs:471-504).  The inverse metric uses the closed form of
// a block-diagonal (t,phi)+(r)+(theta) matrix, which is what nalgebra's
// general inverse computes for these tensors up to rounding.
template <class M>
void numerical_christoffel(const M& metric, const V4<double>& pos, double h,
                           double gamma[4][4][4]) {
  double dg[4][4][4];
  for (int s = 0; s < 4; ++s) {
    V4<double> pp = pos, pm = pos;
    pp[s] += h;
    pm[s] -= h;
    G<double> gp = metric.metric_tensor(pp), gmn = metric.metric_tensor(pm);
    double fp[4][4] = {{gp.tt, 0, 0, gp.tph}, {0, gp.rr, 0, 0}, {0, 0, gp.thth, 0},
                       {gp.tph, 0, 0, gp.phph}};
    double fm[4][4] = {{gmn.tt, 0, 0, gmn.tph}, {0, gmn.rr, 0, 0}, {0, 0, gmn.thth, 0},
                       {gmn.tph, 0, 0, gmn.phph}};
    for (int mu = 0; mu < 4; ++mu)
      for (int nu = 0; nu < 4; ++nu) dg[s][mu][nu] = (fp[mu][nu] - fm[mu][nu]) / (2.0 * h);
  }
  G<double> g = metric.metric_tensor(pos);
  double det = g.tt * g.phph - g.tph * g.tph;
  double gi[4][4] = {{g.phph / det, 0, 0, -g.tph / det},
                     {0, 1.0 / g.rr, 0, 0},
                     {0, 0, 1.0 / g.thth, 0},
                     {-g.tph / det, 0, 0, g.tt / det}};
  for (int mu = 0; mu < 4; ++mu)
    for (int al = 0; al < 4; ++al)
      for (int be = 0; be < 4; ++be) {
        double sum = 0.0;
        for (int s = 0; s < 4; ++s)
          sum += gi[mu][s] * (dg[al][s][be] + dg[be][s][al] - dg[s][al][be]);
        gamma[mu][al][be] = 0.5 * sum;
      }
}

// ---------------------------------------------------------------------------
// Integrators (crates/gr-core/src/geodesic.rs)
// ---------------------------------------------------------------------------
enum StepResult { kContinue = 0, kHorizon = 1, kEscaped = 2, kSingular = 3 };

template <class T>
struct State {
  V4<T> position;
  V4<T> velocity;
  T lambda;
};

template <class T>
inline bool is_valid_position(const V4<T>& pos) {  // :332-334
  using std::isfinite;
  return isfinite(pos[0]) && isfinite(pos[1]) && isfinite(pos[2]) && isfinite(pos[3]) &&
         pos[1] > T(0.0);
}

template <class T>
inline void normalize_spherical_coords(V4<T>& pos) {  // :337-352
  if (pos[2] < T(0.0)) {
    pos[2] = -pos[2];
    pos[3] = pos[3] + T(kPi);
  }
  if (pos[2] > T(kPi)) {
    pos[2] = T(2.0 * kPi) - pos[2];
    pos[3] = pos[3] + T(kPi);
  }
  pos[3] = rem_euclid(pos[3], 2.0 * kPi);
}

// RK4Integrator (:47-152); only the reference's tests use it.
struct RK4 {
  double step_size = 0.1, max_radius = 100.0, horizon_buffer = 0.01;

  template <class M>
  StepResult step(const M& metric, State<double>& st) const {
    double h = step_size;
    V4<double> pos = st.position, vel = st.velocity;
    if (pos[1] > max_radius) return kEscaped;
    double rh;
    if (metric.event_horizon(&rh)) {
      if (pos[1] < rh + horizon_buffer) return kHorizon;
      if (pos[1] < rh) return kHorizon;
    }
    V4<double> k1_pos = vel;
    V4<double> k1_vel = metric.geodesic_acceleration(pos, vel);
    V4<double> pos2 = pos + (0.5 * h) * k1_pos;
    V4<double> vel2 = vel + (0.5 * h) * k1_vel;
    if (!is_valid_position(pos2)) return kSingular;
    V4<double> k2_pos = vel2;
    V4<double> k2_vel = metric.geodesic_acceleration(pos2, vel2);
    V4<double> pos3 = pos + (0.5 * h) * k2_pos;
    V4<double> vel3 = vel + (0.5 * h) * k2_vel;
    if (!is_valid_position(pos3)) return kSingular;
    V4<double> k3_pos = vel3;
    V4<double> k3_vel = metric.geodesic_acceleration(pos3, vel3);
    V4<double> pos4 = pos + h * k3_pos;
    V4<double> vel4 = vel + h * k3_vel;
    if (!is_valid_position(pos4)) return kSingular;
    V4<double> k4_pos = vel4;
    V4<double> k4_vel = metric.geodesic_acceleration(pos4, vel4);
    st.position = pos + (h / 6.0) * (k1_pos + 2.0 * k2_pos + 2.0 * k3_pos + k4_pos);
    st.velocity = vel + (h / 6.0) * (k1_vel + 2.0 * k2_vel + 2.0 * k3_vel + k4_vel);
    st.lambda += h;
    normalize_spherical_coords(st.position);
    return kContinue;
  }
};

// RK45Integrator (:155-329) with the EXTENSION rtol/atol error norm.
struct RK45 {
  double initial_step = 0.1, min_step = 1e-8, max_step = 1.0, tolerance = 1e-6,
         max_radius = 100.0, horizon_buffer = 0.01;
  // EXTENSION: rtol > 0 replaces err = |new_vel - vel_err| and `tolerance`
  // by an RMS norm of the same difference scaled per component by
  // atol + rtol * max(|vel_i|, |new_vel_i|), compared against 1.
  double rtol = 0.0, atol = 0.0;
  // EXTENSION: stepper 1 is the full Dormand-Prince method on the 8-component
  // state (see step_dp45); 0 is the reference's step.
  int stepper = 0;

  // One attempt.  `accepted` (optional) reports whether the state advanced.
  // k_ends (optional, 32 doubles) receives, for an accepted full
  // Dormand-Prince step, its seven stage accelerations k_1..k_7 (4 each,
  // k_7 = a at the new state) and its un-normalised end position, for the
  // crossing interpolant (dense_build).
  template <class M, class T>
  StepResult step(const M& metric, State<T>& st, T& h, bool* accepted = nullptr,
                  T* h_used = nullptr, T* k_ends = nullptr) const {
    if (stepper == 1) return step_dp45(metric, st, h, accepted, h_used, k_ends);
    using std::fabs;
    using std::pow;
    using std::sqrt;
    if (accepted) *accepted = false;
    V4<T> pos = st.position, vel = st.velocity;
    if (pos[1] > T(max_radius)) return kEscaped;
    double rh;
    if (metric.event_horizon(&rh)) {
      if (pos[1] < T(rh + horizon_buffer)) return kHorizon;
    }
    if (metric.event_horizon(&rh) && pos[1] < T(rh)) return kHorizon;

    const T a2(1.0 / 5.0), a3(3.0 / 10.0), a4(4.0 / 5.0), a5(8.0 / 9.0);
    const T b21(1.0 / 5.0), b31(3.0 / 40.0), b32(9.0 / 40.0), b41(44.0 / 45.0),
        b42(-56.0 / 15.0), b43(32.0 / 9.0), b51(19372.0 / 6561.0), b52(-25360.0 / 2187.0),
        b53(64448.0 / 6561.0), b54(-212.0 / 729.0), b61(9017.0 / 3168.0), b62(-355.0 / 33.0),
        b63(46732.0 / 5247.0), b64(49.0 / 176.0), b65(-5103.0 / 18656.0);
    const T c1(35.0 / 384.0), c3(500.0 / 1113.0), c4(125.0 / 192.0), c5(-2187.0 / 6784.0),
        c6(11.0 / 84.0);
    const T d1(5179.0 / 57600.0), d3(7571.0 / 16695.0), d4(393.0 / 640.0),
        d5(-92097.0 / 339200.0), d6(187.0 / 2100.0), d7(1.0 / 40.0);

    V4<T> k1 = metric.geodesic_acceleration(pos, vel);
    V4<T> pos2 = pos + (h * a2) * vel;
    V4<T> vel2 = vel + (h * b21) * k1;
    if (!is_valid_position(pos2)) { h = h * T(0.5); return kContinue; }
    V4<T> k2 = metric.geodesic_acceleration(pos2, vel2);
    V4<T> pos3 = pos + (h * a3) * vel;
    V4<T> vel3 = vel + h * (b31 * k1 + b32 * k2);
    if (!is_valid_position(pos3)) { h = h * T(0.5); return kContinue; }
    V4<T> k3 = metric.geodesic_acceleration(pos3, vel3);
    V4<T> pos4 = pos + (h * a4) * vel;
    V4<T> vel4 = vel + h * (b41 * k1 + b42 * k2 + b43 * k3);
    if (!is_valid_position(pos4)) { h = h * T(0.5); return kContinue; }
    V4<T> k4 = metric.geodesic_acceleration(pos4, vel4);
    V4<T> pos5 = pos + (h * a5) * vel;
    V4<T> vel5 = vel + h * (b51 * k1 + b52 * k2 + b53 * k3 + b54 * k4);
    if (!is_valid_position(pos5)) { h = h * T(0.5); return kContinue; }
    V4<T> k5 = metric.geodesic_acceleration(pos5, vel5);
    V4<T> pos6 = pos + h * vel;
    V4<T> vel6 = vel + h * (b61 * k1 + b62 * k2 + b63 * k3 + b64 * k4 + b65 * k5);
    if (!is_valid_position(pos6)) { h = h * T(0.5); return kContinue; }
    V4<T> k6 = metric.geodesic_acceleration(pos6, vel6);
    V4<T> new_vel = vel + h * (c1 * k1 + c3 * k3 + c4 * k4 + c5 * k5 + c6 * k6);
    V4<T> k7 = metric.geodesic_acceleration(pos6, new_vel);
    V4<T> vel_err = vel + h * (d1 * k1 + d3 * k3 + d4 * k4 + d5 * k5 + d6 * k6 + d7 * k7);

    T err, tol;
    if (rtol > 0.0) {
      // EXTENSION: scaled RMS norm against 1.
      V4<T> diff = new_vel - vel_err;
      T s = T(0.0);
      for (int i = 0; i < 4; ++i) {
        T sc = T(atol) + T(rtol) * rmax(fabs(vel[i]), fabs(new_vel[i]));
        T q = diff[i] / sc;
        s = s + q * q;
      }
      err = sqrt(s * T(0.25));
      tol = T(1.0);
    } else {
      err = norm(new_vel - vel_err);  // :308
      tol = T(tolerance);
    }

    if (err < tol || h <= T(min_step)) {  // :310-321
      st.position = pos + h * vel;
      st.velocity = new_vel;
      st.lambda = st.lambda + h;
      normalize_spherical_coords(st.position);
      if (accepted) *accepted = true;
      if (h_used) *h_used = h;
      if (err > T(0.0)) h = rclamp(h * T(0.9) * pow(tol / err, T(0.2)), min_step, max_step);
    } else {  // :322-325
      h = rmax(h * T(0.9) * pow(tol / err, T(0.25)), T(min_step));
    }
    return kContinue;
  }

  // EXTENSION: the full Dormand-Prince RK5(4) method on y = (x, v), y' =
  // (v, a(x, v)): stage positions use the stage velocities (the reference
  // moves positions along the step's initial velocity only, geodesic.rs:248,
  // 312), the 5th-order solution advances x and v, and the embedded error
  // h * sum_j (c_j - d_j) F_j covers all eight components.  Termination
  // tests, invalid-stage halving, the acceptance test and the step-size law
  // are the reference's (geodesic.rs:195-207, 250-290, 310-325); with rtol > 0
  // the norm is the RMS of the components scaled by atol + rtol*max(|y|,|y'|).
  template <class M, class T>
  StepResult step_dp45(const M& metric, State<T>& st, T& h, bool* accepted, T* h_used,
                       T* k_ends) const {
    using std::fabs;
    using std::pow;
    using std::sqrt;
    if (accepted) *accepted = false;
    const V4<T> x = st.position, v = st.velocity;
    if (x[1] > T(max_radius)) return kEscaped;
    double rh;
    if (metric.event_horizon(&rh) && (x[1] < T(rh + horizon_buffer) || x[1] < T(rh)))
      return kHorizon;

    const double B[7][6] = {
        {0, 0, 0, 0, 0, 0},
        {1.0 / 5.0, 0, 0, 0, 0, 0},
        {3.0 / 40.0, 9.0 / 40.0, 0, 0, 0, 0},
        {44.0 / 45.0, -56.0 / 15.0, 32.0 / 9.0, 0, 0, 0},
        {19372.0 / 6561.0, -25360.0 / 2187.0, 64448.0 / 6561.0, -212.0 / 729.0, 0, 0},
        {9017.0 / 3168.0, -355.0 / 33.0, 46732.0 / 5247.0, 49.0 / 176.0, -5103.0 / 18656.0, 0},
        {35.0 / 384.0, 0.0, 500.0 / 1113.0, 125.0 / 192.0, -2187.0 / 6784.0, 11.0 / 84.0}};
    // 5th-order weights c (= the last row of B) and embedded 4th-order d
    const double D[7] = {5179.0 / 57600.0, 0.0, 7571.0 / 16695.0, 393.0 / 640.0,
                         -92097.0 / 339200.0, 187.0 / 2100.0, 1.0 / 40.0};
    // dw[s] = w[s] - v, kept apart: the weights of the error estimate sum to
    // zero, and summing e_j * w_j instead would leave a rounding floor of
    // eps * |v| in the position error (it steers the step size when the true
    // error is below it, e.g. on long escaping flights)
    V4<T> w[7], dw[7], k[7], xs = x;
    w[0] = v;
    dw[0] = V4<T>{{T(0), T(0), T(0), T(0)}};
    k[0] = metric.geodesic_acceleration(x, v);
    for (int s = 1; s < 7; ++s) {
      V4<T> sx{{T(0), T(0), T(0), T(0)}}, sv{{T(0), T(0), T(0), T(0)}};
      for (int j = 0; j < s; ++j) {
        sx = sx + T(B[s][j]) * w[j];
        sv = sv + T(B[s][j]) * k[j];
      }
      xs = x + h * sx;
      dw[s] = h * sv;
      w[s] = v + dw[s];
      if (!is_valid_position(xs)) {
        h = h * T(0.5);
        return kContinue;
      }
      k[s] = metric.geodesic_acceleration(xs, w[s]);  // s = 6: at the new state (FSAL)
    }
    // xs, w[6] are the 5th-order solution; errors from the weight differences
    V4<T> ex{{T(0), T(0), T(0), T(0)}}, ev{{T(0), T(0), T(0), T(0)}};
    for (int j = 0; j < 7; ++j) {
      const T e = T((j < 6 ? B[6][j] : 0.0) - D[j]);
      ex = ex + e * dw[j];
      ev = ev + e * k[j];
    }
    ex = h * ex;
    ev = h * ev;
    const V4<T> xn = xs, vn = w[6];
    T err, tol;
    if (rtol > 0.0) {
      T s2 = T(0.0);
      for (int i = 0; i < 4; ++i) {
        const T qx = ex[i] / (T(atol) + T(rtol) * rmax(fabs(x[i]), fabs(xn[i])));
        const T qv = ev[i] / (T(atol) + T(rtol) * rmax(fabs(v[i]), fabs(vn[i])));
        s2 = s2 + qx * qx + qv * qv;
      }
      err = sqrt(s2 * T(0.125));
      tol = T(1.0);
    } else {
      err = sqrt(norm(ex) * norm(ex) + norm(ev) * norm(ev));
      tol = T(tolerance);
    }
    if (err < tol || h <= T(min_step)) {
      if (k_ends) {
        for (int j = 0; j < 7; ++j)
          for (int i = 0; i < 4; ++i) k_ends[4 * j + i] = k[j][i];
        for (int i = 0; i < 4; ++i) k_ends[28 + i] = xn[i];
      }
      st.position = xn;
      st.velocity = vn;
      st.lambda = st.lambda + h;
      normalize_spherical_coords(st.position);
      if (accepted) *accepted = true;
      if (h_used) *h_used = h;
      if (err > T(0.0)) h = rclamp(h * T(0.9) * pow(tol / err, T(0.2)), min_step, max_step);
    } else {
      h = rmax(h * T(0.9) * pow(tol / err, T(0.25)), T(min_step));
    }
    return kContinue;
  }
};

// EXTENSION: the continuous extension of the Dormand-Prince pair (Shampine
// 1986; Hairer, Norsett & Wanner, Solving ODEs I, sec. II.6), a 4th-order
// polynomial through an accepted step, used to locate and state the escape
// sphere and disk plane crossings.  With y = (x, v), F_j = (w_j, k_j) the
// stage derivatives (w_j stage velocities, k_j accelerations) and s in
// [0, 1]:  y(s) = y0 + s (r2 + (1-s) (r3 + s (r4 + (1-s) r5))) with
// r2 = y1 - y0, r3 = h F_1 - r2, r4 = r2 - h F_7 - r3, r5 = h sum_j d_j F_j.
// The d_j sum to zero, so the position part of r5 is h sum_j d_j (w_j - v):
// formed from the stage velocity increments, without cancellation.
struct DenseStep {
  double y0[8], r2[8], r3[8], r4[8], r5[8];
};

inline const double* dense_weights() {
  static const double d[7] = {-12715105075.0 / 11282082432.0, 0.0,
                              87487479700.0 / 32700410799.0, -10690763975.0 / 1880347072.0,
                              701980252875.0 / 199316789632.0, -1453857185.0 / 822651844.0,
                              69997945.0 / 29380423.0};
  return d;
}

// xb, vb: start state; xa, va: end state before angle normalisation; k: the
// step's k_1..k_7 (7 x 4); h: the step.
inline void dense_build(const double xb[4], const double vb[4], const double xa[4],
                        const double va[4], const double* k, double h, DenseStep& D) {
  const double B[7][6] = {
      {0, 0, 0, 0, 0, 0},
      {1.0 / 5.0, 0, 0, 0, 0, 0},
      {3.0 / 40.0, 9.0 / 40.0, 0, 0, 0, 0},
      {44.0 / 45.0, -56.0 / 15.0, 32.0 / 9.0, 0, 0, 0},
      {19372.0 / 6561.0, -25360.0 / 2187.0, 64448.0 / 6561.0, -212.0 / 729.0, 0, 0},
      {9017.0 / 3168.0, -355.0 / 33.0, 46732.0 / 5247.0, 49.0 / 176.0, -5103.0 / 18656.0, 0},
      {35.0 / 384.0, 0.0, 500.0 / 1113.0, 125.0 / 192.0, -2187.0 / 6784.0, 11.0 / 84.0}};
  const double* d = dense_weights();
  for (int i = 0; i < 4; ++i) {
    // stage velocity increments w_j - v = h sum_l B[j][l] k_l
    double sw = 0.0, sk = 0.0;
    for (int j = 0; j < 7; ++j) {
      double dw = 0.0;
      for (int l = 0; l < j && l < 6; ++l) dw = dw + B[j][l] * k[4 * l + i];
      sw = sw + d[j] * (h * dw);
      sk = sk + d[j] * k[4 * j + i];
    }
    D.y0[i] = xb[i];
    D.r2[i] = xa[i] - xb[i];
    D.r3[i] = h * vb[i] - D.r2[i];
    D.r4[i] = D.r2[i] - h * va[i] - D.r3[i];
    D.r5[i] = h * sw;
    D.y0[4 + i] = vb[i];
    D.r2[4 + i] = va[i] - vb[i];
    D.r3[4 + i] = h * k[i] - D.r2[4 + i];
    D.r4[4 + i] = D.r2[4 + i] - h * k[24 + i] - D.r3[4 + i];
    D.r5[4 + i] = h * sk;
  }
}

inline double dense_comp(const DenseStep& D, int c, double s) {
  const double t = 1.0 - s;
  return D.y0[c] + s * (D.r2[c] + t * (D.r3[c] + s * (D.r4[c] + t * D.r5[c])));
}

// d/ds of dense_comp
inline double dense_slope(const DenseStep& D, int c, double s) {
  const double t = 1.0 - s;
  return D.r2[c] + (1.0 - 2.0 * s) * D.r3[c] + s * (2.0 - 3.0 * s) * D.r4[c] +
         2.0 * s * t * (1.0 - 2.0 * s) * D.r5[c];
}

inline void dense_point(const DenseStep& D, double s, double out[8]) {
  for (int c = 0; c < 8; ++c) out[c] = dense_comp(D, c, s);
}

// EXTENSION: fraction s in [0, 1] where component c of the continuous
// extension equals `target`, given that it changes sign across the step:
// Newton steps from the chord's root, kept inside a shrinking bracket
// (bisection when a Newton step leaves it); 30 iterations bound the loop.
inline double dense_root(const DenseStep& D, int c, double target) {
  const double flo = dense_comp(D, c, 0.0) - target;
  const double fhi = dense_comp(D, c, 1.0) - target;
  double lo = 0.0, hi = 1.0;
  double s = flo / (flo - fhi);
  if (!(s >= 0.0 && s <= 1.0)) s = 0.5;
  for (int it = 0; it < 30; ++it) {
    const double fs = dense_comp(D, c, s) - target;
    if (fs == 0.0) break;
    if ((fs < 0.0) == (flo < 0.0)) lo = s; else hi = s;
    const double d = dense_slope(D, c, s);
    double sn = d != 0.0 ? s - fs / d : 0.5 * (lo + hi);
    if (!(sn > lo && sn < hi)) sn = 0.5 * (lo + hi);
    if (std::fabs(sn - s) <= 1e-15) {
      s = sn;
      break;
    }
    s = sn;
  }
  return s;
}

// ---------------------------------------------------------------------------
// Camera and ray initialisation (crates/raytracer/src/curved/{camera,ray}.rs)
// ---------------------------------------------------------------------------
struct Camera {
  V4<double> position;
  V3 look_at, up;
  double fov_y_radians, aspect;

  V3 pixel_direction(double u, double v) const {  // camera.rs:20-29
    V3 forward = normalize(look_at);
    V3 right = normalize(cross(forward, up));
    V3 up2 = normalize(cross(right, forward));
    double half_h = std::tan(fov_y_radians / 2.0);
    double half_w = half_h * aspect;
    return normalize(forward + (u * half_w) * right + (v * half_h) * up2);
  }
};

// GeodesicRay::from_camera (ray.rs:14-61) for an image-plane point (u, v).
template <class M>
State<double> from_camera_uv(const M& metric, const Camera& camera, double u, double v) {
  V3 n = camera.pixel_direction(u, v);
  V4<double> pos = camera.position;
  double theta = pos[2], phi = pos[3];
  double st = std::sin(theta), ct = std::cos(theta);
  double sp = std::sin(phi), cp = std::cos(phi);
  V3 r_hat{{st * cp, st * sp, ct}};
  V3 theta_hat{{ct * cp, ct * sp, -st}};
  V3 phi_hat{{-sp, cp, 0.0}};
  double n_r = dot(n, r_hat), n_t = dot(n, theta_hat), n_p = dot(n, phi_hat);
  G<double> g = metric.metric_tensor(pos);
  double kr = n_r / std::sqrt(g.rr);
  double kth = n_t / std::sqrt(g.thth);
  double kph = n_p / std::sqrt(g.phph);
  double spatial_norm_sq = g.rr * kr * kr + g.thth * kth * kth + g.phph * kph * kph;
  double kt = std::sqrt(-spatial_norm_sq / g.tt);
  State<double> s;
  s.position = pos;
  s.velocity = {{kt, kr, kth, kph}};
  s.lambda = 0.0;
  return s;
}

// Pixel -> (u, v) exactly as ray.rs:22-23.
inline void pixel_uv(uint32_t px, uint32_t py, uint32_t width, uint32_t height, double* u,
                     double* v) {
  *u = ((double)px + 0.5) / (double)width * 2.0 - 1.0;
  *v = 1.0 - ((double)py + 0.5) / (double)height * 2.0;
}

// ---------------------------------------------------------------------------
// Disk, redshift, sky, shading
// ---------------------------------------------------------------------------
struct VolumetricDisk {  // disk.rs:8-31
  double r_inner = 6.0, r_outer = 20.0, scale_height = 1.0, density_0 = 1.0,
         temperature_0 = 1.0;

  double density(const V4<double>& pos) const {  // disk.rs:40-59
    double r = pos[1], theta = pos[2];
    double sin_theta = std::sin(theta), cos_theta = std::cos(theta);
    double cap_r = r * std::fabs(sin_theta);
    double z = r * cos_theta;
    if (cap_r < r_inner || cap_r > r_outer) return 0.0;
    double q = r_inner / cap_r;
    double radial = q * q;
    double vertical = std::exp(-z * z / (2.0 * scale_height * scale_height));
    return density_0 * radial * vertical;
  }
  double emission(const V4<double>& pos) const {  // disk.rs:65-81
    double rho = density(pos);
    if (rho == 0.0) return 0.0;
    double r = pos[1], theta = pos[2];
    double cap_r = r * std::fabs(std::sin(theta));
    if (cap_r < r_inner) return 0.0;
    double temp_proxy = std::pow(r_inner / cap_r, 0.75);
    return rho * rho * temp_proxy;
  }
};

// redshift_factor (tracer.rs:158-183)
template <class M>
double redshift_factor(const M& metric, const V4<double>& pos, const V4<double>& p,
                       double sqrt_neg_gtt_obs) {
  G<double> g = metric.metric_tensor(pos);
  double p_t = g.tt * p[0] + g.tph * p[3];
  double e_obs = rmax(-p_t / sqrt_neg_gtt_obs, 0.0);
  double e_emit;
  V4<double> u;
  if (metric.orbital_four_velocity(pos, &u)) {
    double p_phi = g.tph * p[0] + g.phph * p[3];
    e_emit = rmax(-(p_t * u[0] + p_phi * u[3]), 0.0);
  } else {
    double g_tt_emit = -g.tt;
    e_emit = rmax(g_tt_emit > 0.0 ? -p_t / std::sqrt(g_tt_emit) : 0.0, 0.0);
  }
  return e_emit > 0.0 ? e_obs / e_emit : 0.0;
}

inline V3 spatial_dir(const V4<double>& v) {  // tracer.rs:185-189
  V3 s{{v[1], v[2], v[3]}};
  double n = norm(s);
  if (n > 0.0) return {{s[0] / n, s[1] / n, s[2] / n}};
  return {{1.0, 0.0, 0.0}};
}

// ProceduralSky::sample (sky.rs:26-40)
inline void procedural_sky(const V3& dir, double rgb[3]) {
  auto hash = [](double x) -> uint64_t {
    uint64_t bits;
    std::memcpy(&bits, &x, 8);
    return bits * 6364136223846793005ULL + 1442695040888963407ULL;
  };
  auto rotl = [](uint64_t x, int k) -> uint64_t { return (x << k) | (x >> (64 - k)); };
  uint64_t h = hash(dir[0]) ^ rotl(hash(dir[1]), 17) ^ rotl(hash(dir[2]), 34);
  if (h % 512 < 3) {
    double b = (double)(180u + (uint32_t)(h % 75)) / 255.0;
    rgb[0] = rgb[1] = rgb[2] = b;
  } else {
    double v = std::fabs(dir[2]) * 15.0 / 255.0;
    rgb[0] = 0.0;
    rgb[1] = 0.0;
    rgb[2] = 10.0 / 255.0 + v;
  }
}

// EXTENSION: SplitMix64 (Steele, Lea, Flood 2014) finaliser.
inline uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}

// EXTENSION: seeded checkerboard celestial sphere over the escape point's
// (theta, phi): rows x cols cells; light/dark by cell parity, each channel
// scaled by 0.75 + 0.25 u with three 21-bit draws of SplitMix64(seed, cell).
inline void checker_sky(double theta, double phi, uint32_t rows, uint32_t cols, uint64_t seed,
                        double rgb[3]) {
  double cell_h = kPi / (double)rows;
  double cell_w = (2.0 * kPi) / (double)cols;
  double fi = std::floor(theta / cell_h);
  double fj = std::floor(phi / cell_w);
  int64_t i = fi < 0.0 ? 0 : (fi > (double)(rows - 1) ? (int64_t)rows - 1 : (int64_t)fi);
  int64_t j = fj < 0.0 ? 0 : (fj > (double)(cols - 1) ? (int64_t)cols - 1 : (int64_t)fj);
  uint64_t z = splitmix64(seed ^ splitmix64((uint64_t)i * (uint64_t)cols + (uint64_t)j));
  double base = ((i + j) & 1) ? 0.9 : 0.1;
  for (int k = 0; k < 3; ++k) {
    double uk = (double)((z >> (21 * k)) & 0x1FFFFFULL) * (1.0 / 2097152.0);
    rgb[k] = base * (0.75 + 0.25 * uk);
  }
}

// HdriSky (sky.rs:43-123): equirectangular linear RGB f32 texels, row 0 at
// the +z pole, bilinear with wrap in x and clamp in y, scaled by intensity.
struct HdriMap {
  const float* px = nullptr;  // width * height * 3, row-major
  uint32_t width = 0, height = 0;
  float intensity = 1.f;
};

// HdriSky::fetch (sky.rs:85-105)
inline void hdri_fetch(const HdriMap& m, double u, double v, float out[3]) {
  const double w = (double)m.width, h = (double)m.height;
  double fx = std::fmod(u * w, w);  // rem_euclid
  if (fx < 0.0) fx += w;
  double fy = v * h;
  if (fy < 0.0) fy = 0.0;
  if (fy > h - 1.0) fy = h - 1.0;
  const size_t x0 = (size_t)std::floor(fx) % m.width;
  const size_t y0 = (size_t)std::floor(fy);
  const size_t x1 = (x0 + 1) % m.width;
  const size_t y1 = y0 + 1 < m.height ? y0 + 1 : m.height - 1;
  const float tx = (float)(fx - std::floor(fx));
  const float ty = (float)(fy - std::floor(fy));
  auto at = [&](size_t y, size_t x, int c) { return m.px[3 * (y * m.width + x) + c]; };
  auto lerp = [](float a, float b, float t) {
    volatile float d = b - a;  // no contraction into an fma
    volatile float p = d * t;
    return a + p;
  };
  for (int c = 0; c < 3; ++c)
    out[c] = lerp(lerp(at(y0, x0, c), at(y0, x1, c), tx), lerp(at(y1, x0, c), at(y1, x1, c), tx),
                  ty);
}

// HdriSky::sample (sky.rs:108-122)
inline void hdri_sky(const HdriMap& m, const V3& dir, double rgb[3]) {
  double z = dir[2];
  if (z < -1.0) z = -1.0;
  if (z > 1.0) z = 1.0;
  const double theta = std::acos(z);
  const double phi = std::atan2(dir[1], dir[0]);
  constexpr double kFrac1Pi = 0.318309886183790671538;
  const double u = phi * kFrac1Pi * 0.5 + 0.5;
  const double v = theta * kFrac1Pi;
  float px[3];
  hdri_fetch(m, u, v, px);
  for (int c = 0; c < 3; ++c) {
    volatile float s = px[c] * m.intensity;
    rgb[c] = (double)s;
  }
}

// ---------------------------------------------------------------------------
// Objects in the spatial slice (render_with_scene).
// ---------------------------------------------------------------------------
enum ObjKind { kObjSphere = 0, kObjQuad = 1 };
enum MatKind { kMatLambertian = 0, kMatDiffuseLight = 1, kMatMetal = 2, kMatDielectric = 3 };

struct SceneObj {
  int kind = kObjSphere, material = kMatLambertian;
  V3 center{}, q{}, u{}, v{};
  double radius = 1.0;
  V3 color{};  // Lambertian / Metal albedo, DiffuseLight emission
  // Quad::with_arc_material (quad.rs:36-79)
  V3 normal{}, e_alpha{}, e_beta{};
  double d = 0.0;
};

inline V3 sub3(const V3& a, const V3& b) { return {{a[0] - b[0], a[1] - b[1], a[2] - b[2]}}; }

inline SceneObj make_quad(const V3& q, const V3& u, const V3& v, int material, const V3& color) {
  SceneObj o;
  o.kind = kObjQuad;
  o.material = material;
  o.q = q;
  o.u = u;
  o.v = v;
  o.color = color;
  V3 n = cross(u, v);
  o.normal = normalize(n);
  o.d = dot(o.normal, q);
  double nn = dot(n, n);
  V3 w{{n[0] / nn, n[1] / nn, n[2] / nn}};
  o.e_alpha = cross(v, w);
  o.e_beta = cross(w, u);
  return o;
}

struct Hit {
  double t = 0.0;
  V3 point{}, normal{};
  bool front_face = false;
  const SceneObj* obj = nullptr;
};

// HitRecord::new (core/hit.rs): the normal faces the incoming ray
inline void set_face(Hit& h, const V3& dir, const V3& outward) {
  h.front_face = dot(dir, outward) < 0.0;
  h.normal = h.front_face ? outward : V3{{-outward[0], -outward[1], -outward[2]}};
}

// Sphere::hit (sphere.rs:53-87)
inline bool sphere_hit(const SceneObj& s, const V3& o, const V3& dir, double t_min, double t_max,
                       Hit& h) {
  V3 oc = sub3(o, s.center);
  double a = dot(dir, dir);
  double half_b = dot(oc, dir);
  double c = dot(oc, oc) - s.radius * s.radius;
  double disc = half_b * half_b - a * c;
  if (disc < 0.0) return false;
  double sq = std::sqrt(disc);
  double root = (-half_b - sq) / a;
  if (!(t_min < root && root < t_max)) {
    root = (-half_b + sq) / a;
    if (!(t_min < root && root < t_max)) return false;
  }
  h.t = root;
  h.point = o + root * dir;
  V3 diff = sub3(h.point, s.center);
  set_face(h, dir, V3{{diff[0] / s.radius, diff[1] / s.radius, diff[2] / s.radius}});
  h.obj = &s;
  return true;
}

// Quad::hit (quad.rs:85-125)
inline bool quad_hit(const SceneObj& s, const V3& o, const V3& dir, double t_min, double t_max,
                     Hit& h) {
  double denom = dot(s.normal, dir);
  if (std::fabs(denom) < 1e-8) return false;
  double t = (s.d - dot(s.normal, o)) / denom;
  if (!(t_min < t && t < t_max)) return false;
  V3 p = o + t * dir;
  V3 planar = sub3(p, s.q);
  double alpha = dot(planar, s.e_alpha);
  double beta = dot(planar, s.e_beta);
  if (alpha < 0.0 || alpha > 1.0 || beta < 0.0 || beta > 1.0) return false;
  h.t = t;
  h.point = p;
  set_face(h, dir, s.normal);
  h.obj = &s;
  return true;
}

// The nearest hit over all objects for t in (t_min, t_max): what
// World::hit (scene/world.rs:69-81) and BvhNode::hit (accel/bvh.rs:184-254)
// both return, the upper bound shrinking to each hit found.
inline bool scene_hit(const std::vector<SceneObj>& objs, const V3& o, const V3& dir,
                      double t_min, double t_max, Hit& best) {
  bool any = false;
  for (const SceneObj& s : objs) {
    Hit h;
    bool hit = s.kind == kObjSphere ? sphere_hit(s, o, dir, t_min, t_max, h)
                                    : quad_hit(s, o, dir, t_min, t_max, h);
    if (hit) {
      best = h;
      t_max = h.t;
      any = true;
    }
  }
  return any;
}

// shade_hit (curved/tracer.rs:369-384) with the material's scatter
// attenuation: Lambertian albedo (lambertian.rs:42-56), DiffuseLight none
// (diffuse_light.rs:22-30), Metal with fuzz 0 its albedo when the mirror
// direction leaves the surface (metal.rs:40-57, reflect :109-111),
// Dielectric white (dielectric.rs:65-95); emission from DiffuseLight only.
inline void shade_hit(const V3& dir, const Hit& h, double lin[3]) {
  const SceneObj& s = *h.obj;
  V3 albedo{{0.0, 0.0, 0.0}}, emission{{0.0, 0.0, 0.0}};
  V3 unit = normalize(dir);
  switch (s.material) {
    case kMatLambertian: albedo = s.color; break;
    case kMatDiffuseLight: emission = s.color; break;
    case kMatMetal: {
      double two_dot = 2.0 * dot(unit, h.normal);
      V3 refl = sub3(unit, two_dot * h.normal);
      if (dot(refl, h.normal) > 0.0) albedo = s.color;
      break;
    }
    default: albedo = V3{{1.0, 1.0, 1.0}}; break;
  }
  V3 neg{{-unit[0], -unit[1], -unit[2]}};
  double nd = rmax(dot(neg, h.normal), 0.0);
  double facing = 0.5 + 0.5 * nd;
  for (int c = 0; c < 3; ++c) lin[c] = albedo[c] * facing + emission[c];
}

// spherical_to_cartesian / cartesian_to_spherical (curved/tracer.rs:11-28)
inline V3 spherical_to_cartesian(const V4<double>& p) {
  double r = p[1], theta = p[2], phi = p[3];
  double st = std::sin(theta);
  return {{r * st * std::cos(phi), r * st * std::sin(phi), r * std::cos(theta)}};
}
inline V4<double> cartesian_to_spherical(const V3& p) {
  double r = rmax(std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]), 1e-10);
  double z = p[2] / r;
  if (z < -1.0) z = -1.0;
  if (z > 1.0) z = 1.0;
  return {{0.0, r, std::acos(z), std::atan2(p[1], p[0])}};
}

// redshift_g4_static (curved/tracer.rs:40-52)
template <class M>
double redshift_g4_static(const M& metric, const V4<double>& pos_emit, double g_tt_obs) {
  double g_tt_emit = -metric.metric_tensor(pos_emit).tt;
  if (g_tt_emit <= 0.0 || g_tt_obs <= 0.0) return 0.0;
  double g = std::sqrt(g_tt_emit / g_tt_obs);
  double g2 = g * g;
  return g2 * g2;
}

inline void disk_color(double intensity, double rgb[3]) {  // renderer.rs:62-66
  double x = intensity / (1.0 + intensity);
  rgb[0] = std::pow(x, 0.5);
  rgb[1] = std::pow(x, 1.2);
  rgb[2] = std::pow(x, 2.5);
}

inline uint8_t encode_channel(double c) {  // renderer.rs:69-80
  if (c < 0.0) c = 0.0;
  if (c > 1.0) c = 1.0;
  double s = c <= 0.0031308 ? 12.92 * c : 1.055 * std::pow(c, 1.0 / 2.4) - 0.055;
  double q = std::round(s * 255.0);
  if (!(q > 0.0)) return 0;  // NaN saturates to 0 like `as u8`
  if (q > 255.0) return 255;
  return (uint8_t)q;
}

// ---------------------------------------------------------------------------
// Tracing one sample.
// ---------------------------------------------------------------------------
enum RayClass { kClsHorizon = 0, kClsEscaped = 1, kClsDisk = 2, kClsMaxSteps = 3, kClsScene = 5 };
enum DiskKind { kDiskNone = 0, kDiskVolumetric = 1, kDiskThin = 2 };
enum SkyKind { kSkyProcedural = 0, kSkyChecker = 1, kSkyHdri = 2 };

struct ThinDisk {  // EXTENSION
  double r_inner = 6.0, r_outer = 20.0, emissivity_index = 3.0;
};

struct TraceSetup {
  RK45 integ;
  uint32_t max_steps = 5000;
  int disk_kind = kDiskNone;
  VolumetricDisk vdisk;
  ThinDisk tdisk;
  int sky = kSkyProcedural;
  uint32_t sky_rows = 18, sky_cols = 36;
  uint64_t sky_seed = 0;
  HdriMap hdri;
  const std::vector<SceneObj>* scene = nullptr;  // render_with_scene when set
};

struct Sample {
  int cls = kClsMaxSteps;
  State<double> st{};
  uint32_t attempts = 0, accepted = 0;
  double intensity = 0.0, color_temp = 0.0;
  double cross[8];  // state at the escape sphere / disk plane, NaN otherwise
  double rgb[3] = {0, 0, 0};
  double scene_rgb[3] = {0, 0, 0};  // RayOutcome::Scene colour
};

inline void fill_nan(double* p, int n) {
  for (int i = 0; i < n; ++i) p[i] = std::nan("");
}

// Linear point on the last accepted step: the reference moves the position
// by h * vel_before (geodesic.rs:312), so position is exactly linear in the
// step fraction s; velocity is interpolated linearly between the ends.
inline void segment_point(const State<double>& before, const V4<double>& raw_after_pos,
                          const V4<double>& vel_after, double s, double out[8]) {
  for (int i = 0; i < 4; ++i) out[i] = before.position[i] + s * (raw_after_pos[i] - before.position[i]);
  for (int i = 0; i < 4; ++i) out[4 + i] = before.velocity[i] + s * (vel_after[i] - before.velocity[i]);
  V4<double> p{{out[0], out[1], out[2], out[3]}};
  normalize_spherical_coords(p);
  for (int i = 0; i < 4; ++i) out[i] = p[i];
}

template <class M>
void shade(const M&, const TraceSetup& S, Sample& o) {  // renderer.rs:44-53
  switch (o.cls) {
    case kClsHorizon: o.rgb[0] = o.rgb[1] = o.rgb[2] = 0.0; break;
    case kClsEscaped:
      if (S.sky == kSkyChecker) {
        // EXTENSION: with the full Dormand-Prince stepper (thin disk or none)
        // the cell is read where the ray met the escape sphere, a point that
        // does not depend on how far the last step overshot it
        const bool at_cross = S.integ.stepper == 1 && S.disk_kind != kDiskVolumetric &&
                              std::isfinite(o.cross[2]);
        const double th = at_cross ? o.cross[2] : o.st.position[2];
        const double ph = at_cross ? o.cross[3] : o.st.position[3];
        checker_sky(th, ph, S.sky_rows, S.sky_cols, S.sky_seed, o.rgb);
      } else if (S.sky == kSkyHdri) {
        hdri_sky(S.hdri, spatial_dir(o.st.velocity), o.rgb);
      } else {
        procedural_sky(spatial_dir(o.st.velocity), o.rgb);
      }
      break;
    case kClsDisk: disk_color(o.intensity, o.rgb); break;
    case kClsScene:
      for (int c = 0; c < 3; ++c) o.rgb[c] = o.scene_rgb[c];
      break;
    default: o.rgb[0] = 0.0; o.rgb[1] = 0.0; o.rgb[2] = 10.0 / 255.0; break;
  }
}

// trace_ray (tracer.rs:54-70), trace_ray_with_disk (tracer.rs:80-152) and the
// EXTENSION thin-disk tracer, selected by S.disk_kind.
template <class M>
Sample trace(const M& metric, const TraceSetup& S, const V4<double>& observer,
             State<double> st) {
  Sample o;
  fill_nan(o.cross, 8);
  double h = S.integ.initial_step;
  double intensity = 0.0, transmission = 1.0;
  const double absorption_coeff = 0.1;
  G<double> gobs = metric.metric_tensor(observer);
  double g_tt_obs = -gobs.tt;
  double sqrt_neg_gtt_obs = std::sqrt(rmax(g_tt_obs, 0.0));
  const double half_pi = kPi / 2.0;

  auto finish = [&](int cls) {
    o.cls = cls;
    o.st = st;
    shade(metric, S, o);
    return o;
  };

  for (uint32_t it = 0; it < S.max_steps; ++it) {
    State<double> before = st;
    bool acc = false;
    double h_used = 0.0;
    double ends[32];  // full DP: the step's k_1..k_7 and raw end position
    StepResult result = S.integ.step(metric, st, h, &acc, &h_used, ends);
    o.attempts += 1;
    if (acc) o.accepted += 1;
    if (S.scene) {
      // trace_ray_with_scene (tracer.rs:218-236) / trace_ray_with_disk_and_scene
      // (:279-310): the step's Cartesian chord against the scene, before the
      // disk; a step that did not move has no chord
      V3 cb = spherical_to_cartesian(before.position);
      V3 ca = spherical_to_cartesian(st.position);
      V3 seg = sub3(ca, cb);
      if (norm(seg) > 0.0) {
        Hit hit;
        if (scene_hit(*S.scene, cb, seg, 0.0, 1.0, hit)) {
          double lin[3];
          shade_hit(seg, hit, lin);
          double g4 = redshift_g4_static(metric, cartesian_to_spherical(hit.point), g_tt_obs);
          if (S.disk_kind == kDiskVolumetric) {
            double dl[3];
            disk_color(intensity, dl);
            for (int c = 0; c < 3; ++c) o.scene_rgb[c] = lin[c] * g4 * transmission + dl[c];
          } else {
            for (int c = 0; c < 3; ++c) o.scene_rgb[c] = lin[c] * g4;
          }
          o.intensity = intensity;
          return finish(kClsScene);
        }
      }
    }
    if (acc) {
      const bool dp45 = S.integ.stepper == 1;
      const double dl = h_used;
      // the raw (un-normalised) end of the step: the reference's Euler segment
      // (geodesic.rs:312), or the full Dormand-Prince solution
      V4<double> raw = before.position + dl * before.velocity;
      if (dp45) raw = V4<double>{{ends[28], ends[29], ends[30], ends[31]}};
      // state at fraction s of the step: exact on the Euler segment, the
      // continuous extension (EXTENSION) for the full Dormand-Prince step
      DenseStep dense;
      bool dense_ready = false;
      auto ensure_dense = [&]() {
        if (!dense_ready)
          dense_build(before.position.c, before.velocity.c, raw.c, st.velocity.c, ends, dl, dense);
        dense_ready = true;
      };
      auto point = [&](double s, double out[8]) {
        if (!dp45) {
          segment_point(before, raw, st.velocity, s, out);
          return;
        }
        ensure_dense();
        dense_point(dense, s, out);
        V4<double> p{{out[0], out[1], out[2], out[3]}};
        normalize_spherical_coords(p);
        for (int i = 0; i < 4; ++i) out[i] = p[i];
      };
      auto root = [&](int c, double target, double linear_s) {
        if (!dp45) return linear_s;
        ensure_dense();
        return dense_root(dense, c, target);
      };
      // escape-sphere crossing on this step (EXTENSION output)
      if (before.position[1] <= S.integ.max_radius && raw[1] > S.integ.max_radius) {
        double s = root(1, S.integ.max_radius,
                        (S.integ.max_radius - before.position[1]) / (raw[1] - before.position[1]));
        point(s, o.cross);
      }
      if (S.disk_kind == kDiskThin) {
        double d_b = before.position[2] - half_pi;
        double d_a = st.position[2] - half_pi;
        bool crossed = (d_b < 0.0 && d_a >= 0.0) || (d_b > 0.0 && d_a <= 0.0);
        if (crossed) {
          double s = root(2, half_pi, d_b / (d_b - d_a));
          double c[8];
          point(s, c);
          double r_c = dp45 ? c[1] : before.position[1] + s * (raw[1] - before.position[1]);
          if (r_c >= S.tdisk.r_inner && r_c <= S.tdisk.r_outer) {
            for (int i = 0; i < 8; ++i) o.cross[i] = c[i];
            o.cross[1] = r_c;
            o.cross[2] = half_pi;
            V4<double> pc{{o.cross[0], r_c, half_pi, o.cross[3]}};
            V4<double> vc{{o.cross[4], o.cross[5], o.cross[6], o.cross[7]}};
            double g = redshift_factor(metric, pc, vc, sqrt_neg_gtt_obs);
            double q = S.tdisk.r_inner / r_c;
            double g2 = g * g;
            o.intensity = (g2 * g2) * std::pow(q, S.tdisk.emissivity_index);
            o.color_temp = g * std::pow(q, 0.75);
            st.position = pc;
            st.velocity = vc;
            st.lambda = before.lambda + s * dl;
            return finish(kClsDisk);
          }
        }
      }
    }
    if (S.disk_kind == kDiskVolumetric) {
      double dlambda = rmax(st.lambda - before.lambda, 0.0);
      if (dlambda > 0.0) {
        V4<double> mid{{0.5 * (before.position[0] + st.position[0]),
                        0.5 * (before.position[1] + st.position[1]),
                        0.5 * (before.position[2] + st.position[2]),
                        0.5 * (before.position[3] + st.position[3])}};
        double rho = S.vdisk.density(mid);
        if (rho > 0.0) {
          double j = S.vdisk.emission(mid);
          V4<double> pm = 0.5 * (before.velocity + st.velocity);
          double g_factor = redshift_factor(metric, mid, pm, sqrt_neg_gtt_obs);
          double g2 = g_factor * g_factor;
          double redshifted = j * (g2 * g2);
          intensity = intensity + redshifted * dlambda * transmission;
          transmission = transmission * std::exp(-rho * dlambda * absorption_coeff);
          if (transmission < 1e-3) {
            o.intensity = intensity;
            o.color_temp = S.vdisk.temperature_0;
            return finish(kClsDisk);
          }
        }
      }
      if (result == kHorizon || result == kSingular || result == kEscaped) {
        if (intensity > 0.0) {
          o.intensity = intensity;
          o.color_temp = S.vdisk.temperature_0;
          return finish(kClsDisk);
        }
        return finish(result == kEscaped ? kClsEscaped : kClsHorizon);
      }
    } else {
      if (result == kHorizon || result == kSingular) return finish(kClsHorizon);
      if (result == kEscaped) return finish(kClsEscaped);
    }
  }
  if (S.disk_kind == kDiskVolumetric && intensity > 0.0) {
    o.intensity = intensity;
    o.color_temp = S.vdisk.temperature_0;
    return finish(kClsDisk);
  }
  return finish(kClsMaxSteps);
}

}  // namespace ggo
