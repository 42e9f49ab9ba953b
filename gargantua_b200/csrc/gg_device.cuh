// gg_device.cuh -- device-side physics of the GR ray path for sm_100a.
//
// One CUDA thread carries one geodesic through gargantua's RK45 stepper
// (crates/gr-core/src/geodesic.rs:185-328).  The ray state lives in
// registers for the whole trace; only the finished outcome goes to HBM.
//
// Formulation vs the reference.  The reference evaluates Kerr's right-hand
// side by filling a dense 4x4x4 Christoffel array from ~15 divisions and
// contracting all 64 entries (crates/gr-core/src/metric.rs:37-52,
// crates/gr-core/src/kerr.rs:100-424).  Here the same 20 non-zero symbols are
// folded into the contraction: the t and phi rows share the two "energy"
// sums E_t, E_phi, the r and theta rows share their g^rr, g^thth factor, and
// all of 1/Sigma, 1/Delta, 1/sin^2 come from one reciprocal.  The result is
// the same function of (x, v) to rounding.  The stepper's control flow
// (termination tests at the start of a step, invalid-stage halving, the
// acceptance test and the step-size law) is the reference's, test for test.
#pragma once

#include <cstdint>

#include "gg_launch.h"
#include "gg_params.h"

namespace gg {

#define GG_DEV __device__ __forceinline__

constexpr double kPi = 3.14159265358979323846;
constexpr double kHalfPi = kPi / 2.0;
constexpr double kTwoPi = 2.0 * kPi;

// Non-contracted double arithmetic, for the few places that must reproduce
// the reference's rounding bit for bit (ray setup, shading, encoding).
GG_DEV double mul_rn(double a, double b) { return __dmul_rn(a, b); }
GG_DEV double add_rn(double a, double b) { return __dadd_rn(a, b); }
GG_DEV double sub_rn(double a, double b) { return __dsub_rn(a, b); }

// ---------------------------------------------------------------------------
// Geodesic right-hand side a^mu = -Gamma^mu_ab v^a v^b, split in two: the
// position-dependent coefficients of the quadratic form (sincos, one
// reciprocal, the metric derivatives and inverse metric) and the cheap
// contraction with a velocity.  RK45's last two stages (k6 at pos6 with the
// stage velocity, k7 at pos6 with the new velocity, geodesic.rs:284-298) share
// the first part.
// ---------------------------------------------------------------------------

// Kerr in Boyer-Lindquist coordinates.  Metric derivatives are the
// reference's (kerr.rs:154-204) with shared factors pulled out and all of
// 1/Sigma, 1/Delta, 1/sin^2 taken from one reciprocal.
template <class T>
struct KerrGeo {
  T dtt_r, dtt_th, drr_r, drr_th, dthth_r, dthth_th, dphph_r, dphph_th, dtph_r, dtph_th;
  T gtt, gtph, gphph;  // inverse metric, (t, phi) block
  T hrr, hthth;        // -g^rr / 2, -g^thth / 2
};

// 1/x: IEEE division in FP64; in the mixed form's FP32 right-hand side the
// fast reciprocal (__fdividef, within 2 ulp), whose arguments there stay in
// the normal range (r is outside the FP64 band, theta away from the poles).
GG_DEV double rcp(double x) { return 1.0 / x; }
GG_DEV float rcp(float x) { return __fdividef(1.0f, x); }

template <class T>
GG_DEV KerrGeo<T> kerr_geometry(T M, T a, T r, T s, T c) {
  KerrGeo<T> G;
  const T r2 = r * r, a2 = a * a, s2 = s * s, c2 = c * c, sc = s * c;
  const T sig = r2 + a2 * c2;
  const T del = (r - T(2) * M) * r + a2;
  const T rho = r2 + a2;
  const T sd = sig * del;
  const T R = rcp(sd * s2);
  const T iSD = s2 * R;  // 1 / (Sigma Delta)
  const T iS = del * iSD;  // 1 / Sigma
  const T iD = sig * iSD;  // 1 / Delta
  const T is2 = sd * R;    // 1 / sin^2
  const T iS2 = iS * iS;
  const T Mr = M * r;
  const T sm2r = a2 * c2 - r2;  // Sigma - 2 r^2
  G.dtt_r = T(2) * M * sm2r * iS2;
  G.dtt_th = T(4) * Mr * a2 * sc * iS2;
  G.drr_r = T(2) * (a2 * (r * s2 + M * c2) - M * r2) * (iD * iD);
  G.drr_th = T(-2) * a2 * sc * iD;
  G.dthth_r = T(2) * r;
  G.dthth_th = T(-2) * a2 * sc;
  G.dphph_r = T(2) * r * s2 + T(2) * M * a2 * (s2 * s2) * sm2r * iS2;
  G.dphph_th = T(2) * rho * sc + T(4) * Mr * a2 * sc * s2 * (sig + rho) * iS2;
  G.dtph_r = T(-2) * M * a * s2 * sm2r * iS2;
  G.dtph_th = T(-4) * Mr * a * sc * rho * iS2;
  const T big_a = rho * rho - a2 * del * s2;
  G.gtt = -big_a * iSD;
  G.gtph = T(-2) * Mr * a * iSD;
  G.gphph = (del - a2 * s2) * iSD * is2;
  G.hrr = T(-0.5) * del * iS;
  G.hthth = T(-0.5) * iS;
  return G;
}

// t and phi rows share the "energy" sums E_t, E_phi; the r and theta rows
// their -g^ii / 2 factor.
template <class T>
GG_DEV void kerr_contract(const KerrGeo<T>& G, const T v[4], T acc[4]) {
  const T vt = v[0], vr = v[1], vth = v[2], vph = v[3];
  const T Et = vr * (G.dtt_r * vt + G.dtph_r * vph) + vth * (G.dtt_th * vt + G.dtph_th * vph);
  const T Ep = vr * (G.dtph_r * vt + G.dphph_r * vph) + vth * (G.dtph_th * vt + G.dphph_th * vph);
  acc[0] = -(G.gtt * Et + G.gtph * Ep);
  acc[3] = -(G.gtph * Et + G.gphph * Ep);
  const T vt2 = vt * vt, vr2 = vr * vr, vth2 = vth * vth, vph2 = vph * vph;
  const T two_tp = T(2) * vt * vph, two_rt = T(2) * vr * vth;
  acc[1] = G.hrr * (G.drr_r * vr2 - G.dtt_r * vt2 - G.dthth_r * vth2 - G.dphph_r * vph2 +
                    G.drr_th * two_rt - G.dtph_r * two_tp);
  acc[2] = G.hthth * (G.dthth_th * vth2 - G.dtt_th * vt2 - G.drr_th * vr2 - G.dphph_th * vph2 +
                      G.dthth_r * two_rt - G.dtph_th * two_tp);
}

// Schwarzschild (schwarzschild.rs:99-140): 9 non-zero symbols, one reciprocal.
template <class T>
struct SchwGeoT {
  T g_t_tr, g_r_tt, g_r_thth, g_r_phph, ir, g_th_phph, g_ph_thph;
};
using SchwGeo = SchwGeoT<double>;

template <class T>
GG_DEV SchwGeoT<T> schw_geometry(T rs, T r, T s, T c) {
  SchwGeoT<T> G;
  const T rmrs = r - rs;
  const T R = rcp(r * rmrs * s);  // 1 / (r (r - rs) sin)
  const T ifd = s * R;            // 1 / (r (r - rs))
  G.ir = rmrs * ifd;              // 1 / r
  const T is = (r * rmrs) * R;    // 1 / sin
  G.g_t_tr = T(0.5) * rs * ifd;
  G.g_r_tt = T(0.5) * rs * rmrs * (G.ir * G.ir * G.ir);
  G.g_r_thth = -rmrs;
  G.g_r_phph = -rmrs * s * s;
  G.g_th_phph = -s * c;
  G.g_ph_thph = c * is;
  return G;
}

template <class T>
GG_DEV void schw_contract(const SchwGeoT<T>& G, const T v[4], T a[4]) {
  const T vt = v[0], vr = v[1], vth = v[2], vph = v[3];
  a[0] = T(-2) * G.g_t_tr * vt * vr;
  a[1] = -G.g_r_tt * vt * vt + G.g_t_tr * vr * vr - G.g_r_thth * vth * vth -
         G.g_r_phph * vph * vph;
  a[2] = T(-2) * G.ir * vr * vth - G.g_th_phph * vph * vph;
  a[3] = T(-2) * G.ir * vr * vph - T(2) * G.g_ph_thph * vth * vph;
}

template <int METRIC>
struct Geometry;

template <>
struct Geometry<kMetricKerr> {
  KerrGeo<double> g;
  GG_DEV void at(const DevParams& P, double r, double th) {
    double s, c;
    sincos(th, &s, &c);
    g = kerr_geometry<double>(P.mass, P.spin, fmax(r, 1e-10), s, c);
  }
  GG_DEV void accel(const double v[4], double a[4]) const { kerr_contract<double>(g, v, a); }
};

template <>
struct Geometry<kMetricSchwarzschild> {
  SchwGeo g;
  GG_DEV void at(const DevParams& P, double r, double th) {
    double s, c;
    sincos(th, &s, &c);
    g = schw_geometry<double>(P.rs, fmax(r, 1e-10), s, c);
  }
  GG_DEV void accel(const double v[4], double a[4]) const { schw_contract<double>(g, v, a); }
};

template <int METRIC>
GG_DEV void rhs(const DevParams& P, double r, double th, const double v[4], double a[4]) {
  Geometry<METRIC> G;
  G.at(P, r, th);
  G.accel(v, a);
}

// ---------------------------------------------------------------------------
// Metric components and the redshift of a Keplerian emitter (used per
// accepted step by the disks, not per stage).
// ---------------------------------------------------------------------------
struct Gmet {
  double tt, rr, thth, phph, tph;
};

template <int METRIC>
GG_DEV Gmet metric_tensor(const DevParams& P, double r_in, double th) {
  const double r = fmax(r_in, 1e-10);
  const double s = sin(th);
  Gmet g;
  if (METRIC == kMetricKerr) {  // kerr.rs:61-94
    const double m = P.mass, a = P.spin, a2 = a * a;
    const double c = cos(th);
    const double sig = r * r + a * a * c * c;
    const double del = r * r - 2.0 * m * r + a * a;
    const double sin2 = s * s;
    g.tt = -(1.0 - 2.0 * m * r / sig);
    g.rr = sig / del;
    g.thth = sig;
    g.phph = (r * r + a2 + 2.0 * m * a2 * r * sin2 / sig) * sin2;
    g.tph = -2.0 * m * a * r * sin2 / sig;
  } else {  // schwarzschild.rs:26-43
    const double f = 1.0 - P.rs / r;
    g.tt = -f;
    g.rr = 1.0 / f;
    g.thth = r * r;
    g.phph = r * r * s * s;
    g.tph = 0.0;
  }
  return g;
}

// redshift_factor (crates/raytracer/src/curved/tracer.rs:158-183) with the
// metric's orbital_four_velocity (schwarzschild.rs:146-153, kerr.rs:439-449)
// and circular_orbit_velocity (metric.rs:82-94).
template <int METRIC>
GG_DEV double redshift_factor(const DevParams& P, double r, double th, const double p[4]) {
  const Gmet g = metric_tensor<METRIC>(P, r, th);
  const double p_t = g.tt * p[0] + g.tph * p[3];
  const double e_obs = fmax(-p_t / P.sqrt_neg_gtt_obs, 0.0);
  bool has_orbit;
  double omega = 0.0;
  if (METRIC == kMetricKerr) {
    has_orbit = r > 0.0;
    if (has_orbit) {
      const double sqrt_m = sqrt(P.mass);
      omega = sqrt_m / (pow(r, 1.5) + P.spin * sqrt_m);
    }
  } else {
    has_orbit = !(r <= 3.0 * P.mass);
    if (has_orbit) omega = sqrt(P.mass / (r * r * r));
  }
  double e_emit = 0.0;
  bool used_orbit = false;
  if (has_orbit) {
    const Gmet go = metric_tensor<METRIC>(P, r, th);
    const double denom = -(go.tt + 2.0 * go.tph * omega + go.phph * omega * omega);
    if (denom > 0.0 && isfinite(denom)) {
      const double u_t = 1.0 / sqrt(denom);
      const double u_p = omega * u_t;
      const double p_phi = g.tph * p[0] + g.phph * p[3];
      e_emit = fmax(-(p_t * u_t + p_phi * u_p), 0.0);
      used_orbit = true;
    }
  }
  if (!used_orbit) {
    const double g_tt_emit = -g.tt;
    e_emit = fmax(g_tt_emit > 0.0 ? -p_t / sqrt(g_tt_emit) : 0.0, 0.0);
  }
  return e_emit > 0.0 ? e_obs / e_emit : 0.0;
}

// ---------------------------------------------------------------------------
// Ray state and one RK45 attempt.
// ---------------------------------------------------------------------------
struct Ray {
  double x[4];
  double v[4];
  double h;
  double lam;
};

enum StepResult { kContinue = 0, kHorizon = 1, kEscaped = 2 };

GG_DEV bool finite4(double a, double b, double c, double d) {
  return isfinite(a) && isfinite(b) && isfinite(c) && isfinite(d);
}

// normalize_spherical_coords (geodesic.rs:337-352)
GG_DEV void normalize_coords(double x[4]) {
  if (x[2] < 0.0) {
    x[2] = -x[2];
    x[3] = x[3] + kPi;
  }
  if (x[2] > kPi) {
    x[2] = kTwoPi - x[2];
    x[3] = x[3] + kPi;
  }
  // phi.rem_euclid(2 pi).  An accepted step moves phi by far less than 2 pi,
  // so the fmod loop is only needed outside (-2 pi, 4 pi); inside, the result
  // is the same number: on [2 pi, 4 pi) fmod returns p - 2 pi, which that
  // subtraction produces exactly (Sterbenz); on (-2 pi, 0) fmod returns p.
  const double p = x[3];
  double m;
  if (p >= 0.0 && p < kTwoPi) {
    m = p;
  } else if (p >= kTwoPi && p < 2.0 * kTwoPi) {
    m = p - kTwoPi;
  } else if (p < 0.0 && p > -kTwoPi) {
    m = p + kTwoPi;
  } else {
    m = fmod(p, kTwoPi);
    if (m < 0.0) m = m + kTwoPi;
  }
  x[3] = m;
}

// x^(1/5) for the step-size law (geodesic.rs:318): a single-precision seed
// refined by two Newton steps on z = x^(-1/5), z <- z (6/5 - x z^5 / 5),
// which needs no division; x^(1/5) = x z^4.  Agrees with pow(x, 0.2) to a
// few ulp on the range where the seed is representable, pow elsewhere.
GG_DEV double fifth_root(double x) {
  if (!(x >= 1e-30 && x <= 1e30)) return pow(x, 0.2);
  double z = (double)__powf((float)x, -0.2f);
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const double z2 = z * z;
    z = z * (1.2 - 0.2 * x * (z2 * z2 * z));
  }
  const double z2 = z * z;
  return x * (z2 * z2);
}

// Dormand-Prince tableau (geodesic.rs:210-242).
struct DP {
  static constexpr double a2 = 1.0 / 5.0, a3 = 3.0 / 10.0, a4 = 4.0 / 5.0, a5 = 8.0 / 9.0;
  static constexpr double b21 = 1.0 / 5.0;
  static constexpr double b31 = 3.0 / 40.0, b32 = 9.0 / 40.0;
  static constexpr double b41 = 44.0 / 45.0, b42 = -56.0 / 15.0, b43 = 32.0 / 9.0;
  static constexpr double b51 = 19372.0 / 6561.0, b52 = -25360.0 / 2187.0,
                          b53 = 64448.0 / 6561.0, b54 = -212.0 / 729.0;
  static constexpr double b61 = 9017.0 / 3168.0, b62 = -355.0 / 33.0, b63 = 46732.0 / 5247.0,
                          b64 = 49.0 / 176.0, b65 = -5103.0 / 18656.0;
  static constexpr double c1 = 35.0 / 384.0, c3 = 500.0 / 1113.0, c4 = 125.0 / 192.0,
                          c5 = -2187.0 / 6784.0, c6 = 11.0 / 84.0;
  static constexpr double d1 = 5179.0 / 57600.0, d3 = 7571.0 / 16695.0, d4 = 393.0 / 640.0,
                          d5 = -92097.0 / 339200.0, d6 = 187.0 / 2100.0, d7 = 1.0 / 40.0;
};

// Stage position pos + (h a_i) vel (the reference moves stage positions
// along the step's initial velocity, geodesic.rs:248-284); returns false
// when the reference's is_valid_position would reject it.
// Uncontracted like the reference's `pos + h*a*vel`, so the last stage's
// position (ha = h) equals the accepted position bit for bit, which is what
// lets k7 serve as the next step's k1.
GG_DEV bool stage_pos(const Ray& R, double ha, double& r, double& th) {
  const double t = add_rn(R.x[0], mul_rn(ha, R.v[0]));
  r = add_rn(R.x[1], mul_rn(ha, R.v[1]));
  th = add_rn(R.x[2], mul_rn(ha, R.v[2]));
  const double ph = add_rn(R.x[3], mul_rn(ha, R.v[3]));
  return finite4(t, r, th, ph) && r > 0.0;
}

// Where the stage derivatives k1..k6 live between the stages of an attempt
// (and k1 between attempts): this thread's column of a block-shared array,
// [stage][component][thread] so a warp's accesses are conflict-free.  Kept
// out of registers, they free 48 registers of the stepping loop for
// occupancy.
struct KStore {
  double (*s)[4][kTraceBlock];  // [7][4][kTraceBlock], declared by the kernel
  GG_DEV double& operator()(int stage, int i) const { return s[stage][i][threadIdx.x]; }
};

// The same store in a per-thread array (local memory).
struct KStoreLocal {
  double (*k)[4];  // [7][4]
  GG_DEV double& operator()(int stage, int i) const { return k[stage][i]; }
};

// v + h (c1 k1 + c3 k3 + c4 k4 + c5 k5 + c6 k6), left to right, uncontracted
// (geodesic.rs:294-295).
GG_DEV double combine5(double v, double h, double k1, double k3, double k4, double k5,
                       double k6) {
  double s = add_rn(mul_rn(DP::c1, k1), mul_rn(DP::c3, k3));
  s = add_rn(s, mul_rn(DP::c4, k4));
  s = add_rn(s, mul_rn(DP::c5, k5));
  s = add_rn(s, mul_rn(DP::c6, k6));
  return add_rn(v, mul_rn(h, s));
}

// v + h (d1 k1 + d3 k3 + d4 k4 + d5 k5 + d6 k6 + d7 k7), likewise (:299-305).
GG_DEV double combine4(double v, double h, double k1, double k3, double k4, double k5,
                       double k6, double k7) {
  double s = add_rn(mul_rn(DP::d1, k1), mul_rn(DP::d3, k3));
  s = add_rn(s, mul_rn(DP::d4, k4));
  s = add_rn(s, mul_rn(DP::d5, k5));
  s = add_rn(s, mul_rn(DP::d6, k6));
  s = add_rn(s, mul_rn(DP::d7, k7));
  return add_rn(v, mul_rn(h, s));
}

// One call of RK45Integrator::step (geodesic.rs:185-328) in FP64.
// Returns the StepResult; `accepted` and `h_used` describe an advance.
template <int METRIC>
//
// `k1_valid` says K(0, .) already holds a(x, v) for the current state: the
// reference's k7 is evaluated at (pos + h vel, new_vel), exactly the state an
// accepted step moves to, so it is the next attempt's k1 (first same as
// last) unless normalisation reflected theta at a pole; a rejected attempt
// leaves the state, and so k1, unchanged.  The reference recomputes k1; the
// values are identical, one right-hand side per attempt cheaper.
GG_DEV int attempt_fp64(const DevParams& P, Ray& R, const KStore& K, bool& k1_valid,
                        bool& accepted, double& h_used) {
  accepted = false;
  if (R.x[1] > P.max_radius) return kEscaped;
  if (P.has_horizon && (R.x[1] < P.rh_plus_buffer || R.x[1] < P.rh)) return kHorizon;

  const double h = R.h;
  double k7[4], nv[4];
  double r = R.x[1], th = R.x[2];
  // The right-hand-side evaluations run as one loop so the RHS code (sincos,
  // reciprocal, ~150 FP64 ops) is emitted once: unrolled, seven copies
  // overflow the instruction cache and warps stall on fetch.  The stage
  // inputs and the k registers are selected per stage by switch arms
  // (warp-uniform branches; all lanes of a warp run the same stage).  The
  // last pass evaluates k6 and k7, which share the position pos6.
  // Warp-uniform first stage: when a refilled lane in the warp needs k1, the
  // whole warp runs stage 0 instead of the attempt diverged, but a lane whose
  // k1 is valid keeps its own (the previous step's k7).  k7 is evaluated at
  // another call site of the contraction, which the compiler may fuse into
  // multiply-adds differently, so a recomputed k1 can differ from it in the
  // last bit; overwriting it would make a ray's result depend on which rays
  // share its warp.
  const int s_first = __any_sync(__activemask(), !k1_valid) ? 0 : 1;
#pragma unroll 1
  for (int s = s_first; s < 6; ++s) {
    double w[4];
    switch (s) {
      case 0:
#pragma unroll
        for (int i = 0; i < 4; ++i) w[i] = R.v[i];
        break;
      case 1:
        if (!stage_pos(R, h * DP::a2, r, th)) { R.h = h * 0.5; return kContinue; }
#pragma unroll
        for (int i = 0; i < 4; ++i) w[i] = R.v[i] + (h * DP::b21) * K(0, i);
        break;
      case 2:
        if (!stage_pos(R, h * DP::a3, r, th)) { R.h = h * 0.5; return kContinue; }
#pragma unroll
        for (int i = 0; i < 4; ++i) w[i] = R.v[i] + h * (DP::b31 * K(0, i) + DP::b32 * K(1, i));
        break;
      case 3:
        if (!stage_pos(R, h * DP::a4, r, th)) { R.h = h * 0.5; return kContinue; }
#pragma unroll
        for (int i = 0; i < 4; ++i)
          w[i] = R.v[i] + h * (DP::b41 * K(0, i) + DP::b42 * K(1, i) + DP::b43 * K(2, i));
        break;
      case 4:
        if (!stage_pos(R, h * DP::a5, r, th)) { R.h = h * 0.5; return kContinue; }
#pragma unroll
        for (int i = 0; i < 4; ++i)
          w[i] = R.v[i] +
                 h * (DP::b51 * K(0, i) + DP::b52 * K(1, i) + DP::b53 * K(2, i) + DP::b54 * K(3, i));
        break;
      default:
        if (!stage_pos(R, h, r, th)) { R.h = h * 0.5; return kContinue; }
#pragma unroll
        for (int i = 0; i < 4; ++i)
          w[i] = R.v[i] + h * (DP::b61 * K(0, i) + DP::b62 * K(1, i) + DP::b63 * K(2, i) +
                               DP::b64 * K(3, i) + DP::b65 * K(4, i));
        break;
    }
    Geometry<METRIC> G;
    G.at(P, r, th);
    double a[4];
    G.accel(w, a);
    switch (s) {
      case 0:
        if (!k1_valid) {
#pragma unroll
          for (int i = 0; i < 4; ++i) K(0, i) = a[i];
          k1_valid = true;  // a rejected attempt leaves the state, so k1 stays
        }
        break;
      case 1:
#pragma unroll
        for (int i = 0; i < 4; ++i) K(1, i) = a[i];
        break;
      case 2:
#pragma unroll
        for (int i = 0; i < 4; ++i) K(2, i) = a[i];
        break;
      case 3:
#pragma unroll
        for (int i = 0; i < 4; ++i) K(3, i) = a[i];
        break;
      case 4:
#pragma unroll
        for (int i = 0; i < 4; ++i) K(4, i) = a[i];
        break;
      default:
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          K(5, i) = a[i];
          nv[i] = combine5(R.v[i], h, K(0, i), K(2, i), K(3, i), K(4, i), K(5, i));
        }
        G.accel(nv, k7);  // k7 at (pos6, new_vel), geodesic.rs:298
        break;
    }
  }

  // err = |new_vel - vel_err| (geodesic.rs:299-308).  The two vectors agree
  // to ~tol, so err is their last few bits: both are formed exactly as the
  // reference groups them, without fused multiply-adds, so that only the
  // (much smaller) differences in the k's reach the step-size law.
  double err, tol;
  if (P.rtol > 0.0) {
    double ssum = 0.0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const double ve = combine4(R.v[i], h, K(0, i), K(2, i), K(3, i), K(4, i), K(5, i), k7[i]);
      const double sc = add_rn(P.atol, mul_rn(P.rtol, fmax(fabs(R.v[i]), fabs(nv[i]))));
      const double q = __ddiv_rn(sub_rn(nv[i], ve), sc);
      ssum = add_rn(ssum, mul_rn(q, q));
    }
    err = __dsqrt_rn(mul_rn(ssum, 0.25));
    tol = 1.0;
  } else {
    double ssum = 0.0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const double ve = combine4(R.v[i], h, K(0, i), K(2, i), K(3, i), K(4, i), K(5, i), k7[i]);
      const double d = sub_rn(nv[i], ve);
      ssum = add_rn(ssum, mul_rn(d, d));
    }
    err = __dsqrt_rn(ssum);
    tol = P.tolerance;
  }

  if (err < tol || h <= P.min_step) {
#pragma unroll
    for (int i = 0; i < 4; ++i) R.x[i] = add_rn(R.x[i], mul_rn(h, R.v[i]));  // geodesic.rs:312
#pragma unroll
    for (int i = 0; i < 4; ++i) R.v[i] = nv[i];
    R.lam = add_rn(R.lam, h);
    const bool reflected = R.x[2] < 0.0 || R.x[2] > kPi;
    normalize_coords(R.x);
    if (!reflected) {
#pragma unroll
      for (int i = 0; i < 4; ++i) K(0, i) = k7[i];
    }
    k1_valid = !reflected;
    accepted = true;
    h_used = h;
    if (err > 0.0) {
      double hn = h * 0.9 * fifth_root(tol / err);
      hn = hn < P.min_step ? P.min_step : (hn > P.max_step ? P.max_step : hn);
      R.h = hn;
    }
  } else {
    // (tol/err)^0.25 as two correctly rounded square roots
    R.h = fmax(h * 0.9 * sqrt(sqrt(tol / err)), P.min_step);
  }
  return kContinue;
}

// ---------------------------------------------------------------------------
// Full Dormand-Prince RK5(4) on y = (x, v) (GG_STEPPER_DP45).
//
// y'' = a(y, y') is second order, so every stage position and the error of
// the positions can be written with the stage accelerations alone (Nystrom
// form): x_s = x + h a_s v + h^2 sum_l Abar[s][l] k_l with Abar = B B,
// x_new = x + h v + h^2 sum_l Cbar_l k_l, and x_new - x_err =
// h^2 sum_l Ebar_l k_l (the plain weights c and d both sum to 1).  No stage
// velocity needs storing; only the k's, which live in shared memory and are
// indexed by the stage loop directly.
// ---------------------------------------------------------------------------
struct DPTable {
  double B[7][7];     // stage velocity: v_s = v + h sum_l B[s][l] k_l (row 6 = c)
  double Abar[7][7];  // stage position, coefficient of h^2 k_l
  double A[7];        // stage node a_s (row sums of B)
  double E[7];        // c - d, velocity error weights
  double Ebar[7];     // position error weights of h^2 k_l
  double D[7];        // continuous extension weights d_j (sum to zero)
  double Dbar[7];     // their position form: sum_j d_j (w_j - v) = h sum_l Dbar_l k_l
};

constexpr DPTable make_dp_table() {
  DPTable t{};
  const double b[7][7] = {
      {0, 0, 0, 0, 0, 0, 0},
      {1.0 / 5.0, 0, 0, 0, 0, 0, 0},
      {3.0 / 40.0, 9.0 / 40.0, 0, 0, 0, 0, 0},
      {44.0 / 45.0, -56.0 / 15.0, 32.0 / 9.0, 0, 0, 0, 0},
      {19372.0 / 6561.0, -25360.0 / 2187.0, 64448.0 / 6561.0, -212.0 / 729.0, 0, 0, 0},
      {9017.0 / 3168.0, -355.0 / 33.0, 46732.0 / 5247.0, 49.0 / 176.0, -5103.0 / 18656.0, 0, 0},
      {35.0 / 384.0, 0.0, 500.0 / 1113.0, 125.0 / 192.0, -2187.0 / 6784.0, 11.0 / 84.0, 0}};
  const double d[7] = {5179.0 / 57600.0, 0.0, 7571.0 / 16695.0, 393.0 / 640.0,
                       -92097.0 / 339200.0, 187.0 / 2100.0, 1.0 / 40.0};
  for (int s = 0; s < 7; ++s) {
    double a = 0.0;
    for (int l = 0; l < 7; ++l) {
      t.B[s][l] = b[s][l];
      a += b[s][l];
      double ab = 0.0;
      for (int j = l + 1; j < s; ++j) ab += b[s][j] * b[j][l];
      t.Abar[s][l] = ab;
    }
    t.A[s] = a;
  }
  for (int l = 0; l < 7; ++l) {
    const double c_l = l < 6 ? b[6][l] : 0.0;
    t.E[l] = c_l - d[l];
    // x_err uses d_j times stage velocities j = 1..7, the 7th being v_new
    // (row 6 of b is c, and c_7 = b[6][6] = 0)
    double eb = 0.0;
    for (int j = l + 1; j < 7; ++j) eb += (b[6][j] - d[j]) * b[j][l];
    t.Ebar[l] = eb;
  }
  // continuous extension of the pair (Shampine 1986; Hairer, Norsett &
  // Wanner, Solving ODEs I, sec. II.6)
  const double dd[7] = {-12715105075.0 / 11282082432.0, 0.0, 87487479700.0 / 32700410799.0,
                        -10690763975.0 / 1880347072.0, 701980252875.0 / 199316789632.0,
                        -1453857185.0 / 822651844.0, 69997945.0 / 29380423.0};
  for (int l = 0; l < 7; ++l) {
    t.D[l] = dd[l];
    double db = 0.0;
    for (int j = l + 1; j < 7; ++j) db += dd[j] * b[j][l];
    t.Dbar[l] = db;
  }
  return t;
}

__constant__ DPTable kDP = make_dp_table();

// State at the end of an accepted full Dormand-Prince step, for the
// crossing interpolant (a at both ends sits in K(0, .) and K(6, .)).
struct StepEnd {
  double xraw[4];  // new position before angle normalisation
};

// One full Dormand-Prince attempt in FP64.  Same contract as attempt_fp64;
// with k1_valid the previous step's last stage (K(6, .), evaluated at the
// accepted state) is copied to K(0, .) first.  KS is where the stage
// derivatives live: KStore (shared memory) or KStoreLocal (this thread's
// local memory, for the differentiable render's one-ray-per-thread kernels).
template <int METRIC, class KS>
GG_DEV int attempt_dp45_fp64(const DevParams& P, Ray& R, const KS& K, bool& k1_valid,
                             bool& k7_pending, bool& accepted, double& h_used, StepEnd& end) {
  accepted = false;
  if (R.x[1] > P.max_radius) return kEscaped;
  if (P.has_horizon && (R.x[1] < P.rh_plus_buffer || R.x[1] < P.rh)) return kHorizon;
  if (k7_pending) {
#pragma unroll
    for (int i = 0; i < 4; ++i) K(0, i) = K(6, i);
    k7_pending = false;
  }
  const double h = R.h, hh = h * h;
  double xn[4], vn[4];
  const int s_first = __any_sync(__activemask(), !k1_valid) ? 0 : 1;
#pragma unroll 1
  for (int s = s_first; s < 7; ++s) {
    double px[4], pw[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      px[i] = R.x[i];
      pw[i] = R.v[i];
    }
    if (s > 0) {
      const double ha = h * kDP.A[s];
#pragma unroll
      for (int i = 0; i < 4; ++i) px[i] = fma(ha, R.v[i], px[i]);
#pragma unroll 1
      for (int l = 0; l < s; ++l) {
        const double cb = hh * kDP.Abar[s][l], cv = h * kDP.B[s][l];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const double kl = K(l, i);
          px[i] = fma(cb, kl, px[i]);
          pw[i] = fma(cv, kl, pw[i]);
        }
      }
      if (!(finite4(px[0], px[1], px[2], px[3]) && px[1] > 0.0)) {
        R.h = h * 0.5;
        return kContinue;
      }
    }
    Geometry<METRIC> G;
    G.at(P, px[1], px[2]);
    double a[4];
    G.accel(pw, a);
#pragma unroll
    for (int i = 0; i < 4; ++i) K(s, i) = a[i];
    if (s == 6) {
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        xn[i] = px[i];
        vn[i] = pw[i];
      }
    }
  }
  // embedded error of positions (h^2 sum Ebar k) and velocities (h sum E k)
  double ex[4] = {0.0, 0.0, 0.0, 0.0}, ev[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 1
  for (int l = 0; l < 7; ++l) {
    const double eb = kDP.Ebar[l], e = kDP.E[l];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const double kl = K(l, i);
      ex[i] = fma(eb, kl, ex[i]);
      ev[i] = fma(e, kl, ev[i]);
    }
  }
  double err, tol;
  double s2 = 0.0;
  if (P.rtol > 0.0) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const double qx = hh * ex[i] / (P.atol + P.rtol * fmax(fabs(R.x[i]), fabs(xn[i])));
      const double qv = h * ev[i] / (P.atol + P.rtol * fmax(fabs(R.v[i]), fabs(vn[i])));
      s2 = s2 + qx * qx + qv * qv;
    }
    err = sqrt(s2 * 0.125);
    tol = 1.0;
  } else {
#pragma unroll
    for (int i = 0; i < 4; ++i) s2 = s2 + (hh * ex[i]) * (hh * ex[i]) + (h * ev[i]) * (h * ev[i]);
    err = sqrt(s2);
    tol = P.tolerance;
  }
  if (err < tol || h <= P.min_step) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      end.xraw[i] = xn[i];
      R.x[i] = xn[i];
      R.v[i] = vn[i];
    }
    R.lam = R.lam + h;
    const bool reflected = R.x[2] < 0.0 || R.x[2] > kPi;
    normalize_coords(R.x);
    // K(6, .) = a(x_new, v_new): the next k1 unless theta was reflected;
    // copied at the next attempt so the caller can still read this step's k1
    k1_valid = !reflected;
    k7_pending = !reflected;
    accepted = true;
    h_used = h;
    if (err > 0.0) {
      double hn = h * 0.9 * fifth_root(tol / err);
      hn = hn < P.min_step ? P.min_step : (hn > P.max_step ? P.max_step : hn);
      R.h = hn;
    }
  } else {
    R.h = fmax(h * 0.9 * sqrt(sqrt(tol / err)), P.min_step);
  }
  return kContinue;
}

// An accepted full Dormand-Prince step, for locating a crossing inside it:
// start state, end state before angle normalisation, step, and the seven
// stage accelerations k_1..k_7 (k_7 = a at the end).  Kernels fill one only
// on the (once per ray) path where a crossing was detected.
struct StepSpan {
  double xb[4], vb[4], xa[4], va[4];
  double k[7][4];
  double h;
};

// Continuous extension of the Dormand-Prince pair (Shampine 1986; Hairer,
// Norsett & Wanner, Solving ODEs I, sec. II.6), a 4th-order polynomial in the
// step fraction s for each of the 8 components of y = (x, v):
// y(s) = y0 + s (r2 + (1-s) (r3 + s (r4 + (1-s) r5))), r2 = y1 - y0,
// r3 = h y'(0) - r2, r4 = r2 - h y'(1) - r3, r5 = h sum_j d_j F_j.  The d_j
// sum to zero, so the position part of r5 is h^2 sum_l Dbar_l k_l.
struct DenseComp {
  double y0, r2, r3, r4, r5;
  GG_DEV double at(double s) const {
    const double t = 1.0 - s;
    return y0 + s * (r2 + t * (r3 + s * (r4 + t * r5)));
  }
  GG_DEV double slope(double s) const {
    const double t = 1.0 - s;
    return r2 + (1.0 - 2.0 * s) * r3 + s * (2.0 - 3.0 * s) * r4 + 2.0 * s * t * (1.0 - 2.0 * s) * r5;
  }
};

GG_DEV DenseComp dense_comp(const StepSpan& sp, int c) {
  DenseComp q;
  double w = 0.0;
  if (c < 4) {
    for (int l = 0; l < 6; ++l) w = fma(kDP.Dbar[l], sp.k[l][c], w);
    q.y0 = sp.xb[c];
    q.r2 = sp.xa[c] - sp.xb[c];
    q.r3 = sp.h * sp.vb[c] - q.r2;
    q.r4 = q.r2 - sp.h * sp.va[c] - q.r3;
    q.r5 = sp.h * sp.h * w;
  } else {
    const int i = c - 4;
    for (int l = 0; l < 7; ++l) w = fma(kDP.D[l], sp.k[l][i], w);
    q.y0 = sp.vb[i];
    q.r2 = sp.va[i] - sp.vb[i];
    q.r3 = sp.h * sp.k[0][i] - q.r2;
    q.r4 = q.r2 - sp.h * sp.k[6][i] - q.r3;
    q.r5 = sp.h * w;
  }
  return q;
}

// Locates where component `comp` of the step's continuous extension meets
// `target` (it changes sign across the step): safeguarded Newton from the
// chord's root inside a shrinking bracket, at most 30 iterations.  Writes the
// 8-component state there (angles not yet normalised) and returns the step
// fraction.  Out of line: once per ray.
static __device__ __noinline__ double dense_crossing(const StepSpan& sp, int comp, double target,
                                              double out[8]) {
  const DenseComp q = dense_comp(sp, comp);
  const double flo = q.at(0.0) - target;
  const double fhi = q.at(1.0) - target;
  double lo = 0.0, hi = 1.0;
  double s = flo / (flo - fhi);
  if (!(s >= 0.0 && s <= 1.0)) s = 0.5;
  for (int it = 0; it < 30; ++it) {
    const double fs = q.at(s) - target;
    if (fs == 0.0) break;
    if ((fs < 0.0) == (flo < 0.0)) lo = s; else hi = s;
    const double d = q.slope(s);
    double sn = d != 0.0 ? s - fs / d : 0.5 * (lo + hi);
    if (!(sn > lo && sn < hi)) sn = 0.5 * (lo + hi);
    if (fabs(sn - s) <= 1e-15) {
      s = sn;
      break;
    }
    s = sn;
  }
  for (int c = 0; c < 8; ++c) out[c] = dense_comp(sp, c).at(s);
  return s;
}

// The same, for a step whose data a source object reads where it lives
// (Src::xb(c), vb(c), xa(c), va(c), k(l, c), h), one component at a time:
// no step record is built.  COMP is the component whose crossing is sought;
// the same arithmetic as dense_comp / dense_crossing, so the same results.
template <class Src>
GG_DEV DenseComp dense_comp_src(const Src& sp, int c) {
  DenseComp q;
  double w = 0.0;
  if (c < 4) {
#pragma unroll
    for (int l = 0; l < 6; ++l) w = fma(kDP.Dbar[l], sp.k(l, c), w);
    q.y0 = sp.xb(c);
    q.r2 = sp.xa(c) - sp.xb(c);
    q.r3 = sp.h * sp.vb(c) - q.r2;
    q.r4 = q.r2 - sp.h * sp.va(c) - q.r3;
    q.r5 = sp.h * sp.h * w;
  } else {
    const int i = c - 4;
#pragma unroll
    for (int l = 0; l < 7; ++l) w = fma(kDP.D[l], sp.k(l, i), w);
    q.y0 = sp.vb(i);
    q.r2 = sp.va(i) - sp.vb(i);
    q.r3 = sp.h * sp.k(0, i) - q.r2;
    q.r4 = q.r2 - sp.h * sp.k(6, i) - q.r3;
    q.r5 = sp.h * w;
  }
  return q;
}

template <int COMP, class Src>
GG_DEV double dense_crossing_src(const Src& sp, double target, double out[8]) {
  const DenseComp q = dense_comp_src(sp, COMP);
  const double flo = q.at(0.0) - target;
  const double fhi = q.at(1.0) - target;
  double lo = 0.0, hi = 1.0;
  double s = flo / (flo - fhi);
  if (!(s >= 0.0 && s <= 1.0)) s = 0.5;
  for (int it = 0; it < 30; ++it) {
    const double fs = q.at(s) - target;
    if (fs == 0.0) break;
    if ((fs < 0.0) == (flo < 0.0)) lo = s; else hi = s;
    const double d = q.slope(s);
    double sn = d != 0.0 ? s - fs / d : 0.5 * (lo + hi);
    if (!(sn > lo && sn < hi)) sn = 0.5 * (lo + hi);
    if (fabs(sn - s) <= 1e-15) {
      s = sn;
      break;
    }
    s = sn;
  }
#pragma unroll
  for (int c = 0; c < 8; ++c) out[c] = dense_comp_src(sp, c).at(s);
  return s;
}

// ---------------------------------------------------------------------------
// Camera rays (crates/raytracer/src/curved/{camera,ray}.rs) with the
// reference's rounding: the camera frame is prepared on the host; here only
// the per-pixel part runs, every operation uncontracted.
// ---------------------------------------------------------------------------
GG_DEV uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}

GG_DEV double jitter_unit(uint64_t seed, uint64_t key) {
  return (double)(splitmix64(seed ^ splitmix64(key)) >> 11) * (1.0 / 9007199254740992.0);
}

// Image-plane (u, v) of global sample `idx` (pixel-major, samples inside).
GG_DEV void sample_uv(const DevParams& P, uint64_t idx, double& u, double& v) {
  const uint64_t pix = idx / P.spp;
  const uint32_t s = (uint32_t)(idx - pix * P.spp);
  const uint32_t prow = (uint32_t)(pix / P.width);  // row among the traced rows
  const uint32_t px = (uint32_t)(pix - (uint64_t)prow * P.width);
  const uint32_t py = P.row0 + prow * P.row_step;   // row of the image
  if (P.jitter_spp > 0) {
    // keyed by the sample's index in the whole image, so a frame split
    // across GPUs jitters every sample as the unsplit frame does
    const uint64_t gidx = ((uint64_t)py * P.width + px) * P.spp + s;
    const double ox = jitter_unit(P.seed, 2 * gidx);
    const double oy = jitter_unit(P.seed, 2 * gidx + 1);
    u = sub_rn(mul_rn(__ddiv_rn(add_rn((double)px, ox), (double)P.width), 2.0), 1.0);
    v = sub_rn(1.0, mul_rn(__ddiv_rn(add_rn((double)py, oy), (double)P.height), 2.0));
    return;
  }
  const uint32_t sy = s / P.spa, sx = s - sy * P.spa;
  const uint32_t spx = px * P.spa + sx, spy = py * P.spa + sy;
  u = sub_rn(mul_rn(__ddiv_rn((double)spx + 0.5, (double)P.sub_w), 2.0), 1.0);
  v = sub_rn(1.0, mul_rn(__ddiv_rn((double)spy + 0.5, (double)P.sub_h), 2.0));
}

GG_DEV double dot3_rn(const double a[3], const double b[3]) {
  return add_rn(add_rn(mul_rn(a[0], b[0]), mul_rn(a[1], b[1])), mul_rn(a[2], b[2]));
}

// GeodesicRay::from_camera (ray.rs:14-61) for image-plane point (u, v).
GG_DEV void init_ray(const DevParams& P, double u, double v, Ray& R) {
  double d[3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
    d[i] = add_rn(add_rn(P.cam_forward[i], mul_rn(mul_rn(u, P.half_w), P.cam_right[i])),
                  mul_rn(mul_rn(v, P.half_h), P.cam_up[i]));
  const double n = __dsqrt_rn(dot3_rn(d, d));
  double dir[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) dir[i] = __ddiv_rn(d[i], n);
  const double n_r = dot3_rn(dir, P.r_hat);
  const double n_t = dot3_rn(dir, P.theta_hat);
  const double n_p = dot3_rn(dir, P.phi_hat);
  const double kr = __ddiv_rn(n_r, P.sqrt_g_rr);
  const double kth = __ddiv_rn(n_t, P.sqrt_g_thth);
  const double kph = __ddiv_rn(n_p, P.sqrt_g_phph);
  const double sns = add_rn(add_rn(mul_rn(mul_rn(P.cam_g_rr, kr), kr),
                                   mul_rn(mul_rn(P.cam_g_thth, kth), kth)),
                            mul_rn(mul_rn(P.cam_g_phph, kph), kph));
  const double kt = __dsqrt_rn(__ddiv_rn(-sns, P.cam_g_tt));
#pragma unroll
  for (int i = 0; i < 4; ++i) R.x[i] = P.cam_pos[i];
  R.v[0] = kt;
  R.v[1] = kr;
  R.v[2] = kth;
  R.v[3] = kph;
  R.lam = 0.0;
  R.h = P.initial_step;
}

// ---------------------------------------------------------------------------
// Shading (crates/raytracer/src/curved/renderer.rs:44-80, sky.rs:26-40).
// ---------------------------------------------------------------------------
// spatial_dir (tracer.rs:185-189): (v^r, v^theta, v^phi) normalised as a
// Cartesian 3-vector, (1, 0, 0) for a zero vector.
GG_DEV void spatial_dir(const double v[4], double& d0, double& d1, double& d2) {
  const double sx = v[1], sy = v[2], sz = v[3];
  const double n = __dsqrt_rn(add_rn(add_rn(mul_rn(sx, sx), mul_rn(sy, sy)), mul_rn(sz, sz)));
  d0 = 1.0;
  d1 = 0.0;
  d2 = 0.0;
  if (n > 0.0) {
    d0 = __ddiv_rn(sx, n);
    d1 = __ddiv_rn(sy, n);
    d2 = __ddiv_rn(sz, n);
  }
}

// HdriSky::sample and fetch (sky.rs:88-123): theta = acos(z), phi =
// atan2(y, x), u = phi / (2 pi) + 1/2, v = theta / pi; bilinear in f32 with
// wrap in x and clamp in y, in the reference's order without contraction.
GG_DEV void hdri_sky(const DevParams& P, const double v[4], double rgb[3]) {
  double d0, d1, d2;
  spatial_dir(v, d0, d1, d2);
  const double z = fmin(fmax(d2, -1.0), 1.0);
  const double theta = acos(z);
  const double phi = atan2(d1, d0);
  constexpr double kFrac1Pi = 0.318309886183790671538;
  const double u = add_rn(mul_rn(mul_rn(phi, kFrac1Pi), 0.5), 0.5);
  const double vv = mul_rn(theta, kFrac1Pi);
  const double w = (double)P.hdri_w, h = (double)P.hdri_h;
  double fx = fmod(mul_rn(u, w), w);
  if (fx < 0.0) fx = add_rn(fx, w);
  const double fy = fmin(fmax(mul_rn(vv, h), 0.0), sub_rn(h, 1.0));
  const uint32_t x0 = (uint32_t)floor(fx) % P.hdri_w;
  const uint32_t y0 = (uint32_t)floor(fy);
  const uint32_t x1 = (x0 + 1) % P.hdri_w;
  const uint32_t y1 = y0 + 1 < P.hdri_h ? y0 + 1 : P.hdri_h - 1;
  const float tx = (float)sub_rn(fx, floor(fx));
  const float ty = (float)sub_rn(fy, floor(fy));
  const float* p00 = P.hdri + 3 * ((uint64_t)y0 * P.hdri_w + x0);
  const float* p10 = P.hdri + 3 * ((uint64_t)y0 * P.hdri_w + x1);
  const float* p01 = P.hdri + 3 * ((uint64_t)y1 * P.hdri_w + x0);
  const float* p11 = P.hdri + 3 * ((uint64_t)y1 * P.hdri_w + x1);
  auto lerp = [](float a, float b, float t) { return __fadd_rn(a, __fmul_rn(__fsub_rn(b, a), t)); };
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float px = lerp(lerp(p00[c], p10[c], tx), lerp(p01[c], p11[c], tx), ty);
    rgb[c] = (double)__fmul_rn(px, P.hdri_intensity);
  }
}

// ProceduralSky::sample (sky.rs:26-40) of a unit direction (d0, d1, d2):
// the hash of the directions' f64 bits picks stars, else a blue gradient.
GG_DEV void procedural_sky_dir(double d0, double d1, double d2, double rgb[3]) {
  auto hash = [](double x) -> uint64_t {
    return (uint64_t)__double_as_longlong(x) * 6364136223846793005ULL +
           1442695040888963407ULL;
  };
  auto rotl = [](uint64_t x, int k) -> uint64_t { return (x << k) | (x >> (64 - k)); };
  const uint64_t h = hash(d0) ^ rotl(hash(d1), 17) ^ rotl(hash(d2), 34);
  if (h % 512 < 3) {
    const double b = (double)(180u + (uint32_t)(h % 75)) / 255.0;
    rgb[0] = rgb[1] = rgb[2] = b;
  } else {
    const double vv = __ddiv_rn(mul_rn(fabs(d2), 15.0), 255.0);
    rgb[0] = 0.0;
    rgb[1] = 0.0;
    rgb[2] = add_rn(10.0 / 255.0, vv);
  }
}

// The starfield seen along an escaped ray's final velocity (tracer.rs:185-189
// then sky.rs:26-40).
GG_DEV void procedural_sky(const double v[4], double rgb[3]) {
  double d0, d1, d2;
  spatial_dir(v, d0, d1, d2);
  procedural_sky_dir(d0, d1, d2, rgb);
}

// Seeded checkerboard over the escape point's (theta, phi).
GG_DEV void checker_sky(const DevParams& P, double theta, double phi, double rgb[3]) {
  const double fi = floor(__ddiv_rn(theta, P.cell_h));
  const double fj = floor(__ddiv_rn(phi, P.cell_w));
  const int64_t i = fi < 0.0 ? 0 : (fi > (double)(P.sky_rows - 1) ? (int64_t)P.sky_rows - 1 : (int64_t)fi);
  const int64_t j = fj < 0.0 ? 0 : (fj > (double)(P.sky_cols - 1) ? (int64_t)P.sky_cols - 1 : (int64_t)fj);
  const uint64_t z = splitmix64(P.sky_seed ^ splitmix64((uint64_t)i * P.sky_cols + (uint64_t)j));
  const double base = ((i + j) & 1) ? 0.9 : 0.1;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double uk = (double)((z >> (21 * k)) & 0x1FFFFFULL) * (1.0 / 2097152.0);
    rgb[k] = mul_rn(base, add_rn(0.75, mul_rn(0.25, uk)));
  }
}

GG_DEV void disk_color(double intensity, double rgb[3]) {  // renderer.rs:62-66
  const double x = __ddiv_rn(intensity, add_rn(1.0, intensity));
  rgb[0] = pow(x, 0.5);
  rgb[1] = pow(x, 1.2);
  rgb[2] = pow(x, 2.5);
}

GG_DEV uint8_t encode_channel(double c) {  // renderer.rs:69-80
  c = c < 0.0 ? 0.0 : (c > 1.0 ? 1.0 : c);
  const double s = c <= 0.0031308 ? mul_rn(12.92, c)
                                  : sub_rn(mul_rn(1.055, pow(c, 1.0 / 2.4)), 0.055);
  const double q = round(mul_rn(s, 255.0));
  if (!(q > 0.0)) return 0;
  if (q > 255.0) return 255;
  return (uint8_t)q;
}

}  // namespace gg
