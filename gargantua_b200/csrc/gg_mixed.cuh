// gg_mixed.cuh -- the mixed-precision form of the full Dormand-Prince step.
//
// Where the precision goes.  The ray state (x, v) is a pair of floats per
// component, hi + lo (about 48 significant bits), and each accepted step adds
// its FP32 increment to it with a compensated (two-sum) addition: without
// that, rounding the state to FP32 every step would cost eps * |x| per step,
// 1e-5 M at r = 200 after a few hundred steps.  Everything that is small
// relative to the state runs in FP32: the stage positions and velocities
// (formed as increments over the state) and the seven right-hand sides.  The
// embedded error estimate -- which the Nystrom form builds directly from the
// stage derivatives (weights c - d), so it carries no cancellation -- is
// summed and normed in FP64, and the step-size controller (acceptance test,
// fifth root, clamps, the step h itself) is FP64.  Attempts that start within
// 0.5 M of the horizon or of the prograde photon orbit, or near a pole (where
// Boyer-Lindquist theta turns and is reflected), run in the FP64 pass: the
// ray is handed over with its state converted to FP64 (gg_mixed.cu).
//
// Where the state lives.  Registers hold only what every stage reads: the
// velocity's hi part and the FP64 step.  The position pair, the velocity's
// lo part, the affine parameter and the sample index live in this lane's
// column of shared memory (MixedSmem), read once per attempt and written
// once per accepted step, which keeps the stepping loop within 64 registers
// without spilling.  The right-hand side depends on (r, theta, v) only -- the
// metric is stationary and axisymmetric -- so stages form r and theta alone;
// the t and phi increments are formed once, for the accepted step.
#pragma once

#include "gg_device.cuh"

// Build knobs of the mixed attempt (tuning builds compare them):
// GG_MIXED_ERR_FP64 (default) forms the embedded error estimate -- its sums
// over the FP32 stage derivatives and its norm -- in FP64; 0 forms the sums in
// FP32 and only the norm's reduction in FP64.  Measured on the 1080p Kerr
// frame: FP64 sums 27.0 ms, FP32 sums 25.4 ms, with the same attempts (416.56
// M against 416.72 M) and the same crossing-error distribution (p50 1.05e-7,
// p99 3.9e-7): the estimate's noise comes from the FP32 stage derivatives
// themselves, which FP64 sums do not remove.  GG_MIXED_STAGE_UNROLL unrolls
// the seven stages instead of looping over one copy of the right-hand side
// (26.2 ms: more spills, not kept).  GG_MIXED_ROOT10 (default) runs the
// acceptance test and the step law on the squared norm s2 itself (s2 < 8;
// h 0.9 (8 / s2)^(1/10)) instead of forming err = sqrt(s2 / 8), tol / err and
// its fifth root: 26.35 against 26.95 ms, the same attempts to 20 in 416.6 M.
// GG_MIXED_PAIRED (default) forms the stage sums with the paired FP32 fused
// multiply-add and the accepted step's two-sum state update with the paired
// add, two components per instruction: 25.7 against 26.5 ms, the same bits.
// Pairing the contraction's r and theta rows the same way (26.6 ms) or the
// stage-6 position increments (26.2 ms) or the polar sine and cosine's two
// Horner chains (26.0 against 25.5 ms) gave the same bits too but cost more
// in register moves, constant pairs and spills than they saved.
#ifndef GG_MIXED_ERR_FP64
#define GG_MIXED_ERR_FP64 1
#endif
#ifndef GG_MIXED_STAGE_UNROLL
#define GG_MIXED_STAGE_UNROLL 0
#endif
#ifndef GG_MIXED_ROOT10
#define GG_MIXED_ROOT10 1
#endif
#ifndef GG_MIXED_PAIRED
#define GG_MIXED_PAIRED 1
#endif

namespace gg {

constexpr float kPiHi = 3.14159274101257324f;  // float(pi), rounded up
constexpr float kPiLo = -8.74227765734758577e-08f;  // pi - kPiHi
constexpr float kHalfPiHi = 1.57079637050628662f;
constexpr float kHalfPiLo = -4.37113882867379300e-08f;  // pi/2 - kHalfPiHi
constexpr float kTwoPiHi = 6.28318548202514648f;
constexpr float kTwoPiLo = -1.74845553146951720e-07f;  // 2 pi - kTwoPiHi
constexpr float kQuarterPiF = 0.785398163397448310f;

// sin and cos of a Boyer-Lindquist polar angle, for theta in [-pi/4, 5pi/4]:
// reduce to |u| <= pi/4 about 0, pi/2 or pi (the reductions about pi/2 and pi
// subtract the float pair of the constant, exactly in its leading part by
// Sterbenz), then the Taylor series of sin u to u^9 and of cos u to u^10
// (truncation below 2e-9 on |u| <= pi/4), Horner with fused multiply-adds.
// Branch-free; the same source runs on the host for testing.
__host__ __device__ __forceinline__ void sincos_polar(float th, float* s_out, float* c_out) {
  const bool lo_q = th < kQuarterPiF;
  const bool hi_q = th > 3.0f * kQuarterPiF;
  const float u_mid = (th - kHalfPiHi) - kHalfPiLo;  // theta = pi/2 + u
  const float u_top = (kPiHi - th) + kPiLo;          // theta = pi - u
  const float u = lo_q ? th : (hi_q ? u_top : u_mid);
  const float u2 = u * u;
  float ps = fmaf(u2, 1.0f / 362880.0f, -1.0f / 5040.0f);
  ps = fmaf(u2, ps, 1.0f / 120.0f);
  ps = fmaf(u2, ps, -1.0f / 6.0f);
  ps = u2 * ps;
  const float su = fmaf(u, ps, u);
  float pc = fmaf(u2, -1.0f / 3628800.0f, 1.0f / 40320.0f);
  pc = fmaf(u2, pc, -1.0f / 720.0f);
  pc = fmaf(u2, pc, 1.0f / 24.0f);
  pc = fmaf(u2, pc, -0.5f);
  const float cu = fmaf(u2, pc, 1.0f);
  *s_out = lo_q ? su : (hi_q ? su : cu);
  *c_out = lo_q ? cu : (hi_q ? -cu : -su);
}

// hi + lo += d: two-sum of hi and d (exact), its rounding error folded into
// lo, then renormalised so that |lo| <= ulp(hi) / 2.
GG_DEV void ff_add(float& hi, float& lo, float d) {
  const float s = hi + d;
  const float bb = s - hi;
  const float e = (hi - (s - bb)) + (d - bb);
  const float t = lo + e;
  hi = s + t;
  lo = t - (hi - s);
}

#if GG_MIXED_PAIRED
// ff_add on two components at once with the paired FP32 add (a - b as
// a + (-b), exact): the same operations per lane, so the same bits.
GG_DEV float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }
GG_DEV void ff_add2(float2& hi, float2& lo, float2 d) {
  const float2 s = __fadd2_rn(hi, d);
  const float2 bb = __fadd2_rn(s, neg2(hi));
  const float2 e =
      __fadd2_rn(__fadd2_rn(hi, neg2(__fadd2_rn(s, neg2(bb)))), __fadd2_rn(d, neg2(bb)));
  const float2 t = __fadd2_rn(lo, e);
  hi = __fadd2_rn(s, t);
  lo = __fadd2_rn(t, neg2(__fadd2_rn(hi, neg2(s))));
}
#endif

// (hi + lo) - (c_hi + c_lo) to FP32 accuracy, exact in its leading part when
// hi is within a factor 2 of c_hi (Sterbenz): the sign tests of the escape
// sphere and the disk plane are made on this difference.
GG_DEV float ff_minus(float hi, float lo, float c_hi, float c_lo) {
  return (hi - c_hi) + (lo - c_lo);
}

GG_DEV void split(double x, float& hi, float& lo) {
  hi = (float)x;
  lo = (float)(x - (double)hi);
}

// This lane's column of the mixed kernel's shared memory: float4 slots
// [slot][thread] (a warp's 16-byte accesses are conflict-free), plus the
// affine parameter and sample index.  Slots 0-6 hold k1..k7 (k7 = a at the
// new state, the next attempt's k1); 7 and 8 the accepted step's increments
// dx, dv; 9 and 10 the position hi and lo parts; 11 the velocity lo part.
constexpr int kSlotDx = 7, kSlotDv = 8, kSlotXh = 9, kSlotXl = 10, kSlotVl = 11;
constexpr int kMixedSlots = 12;
// Shared memory of a CTA of BLOCK threads: the slots, then the affine
// parameters and sample indices.
template <int BLOCK>
constexpr int mixed_smem_bytes() {
  return kMixedSlots * BLOCK * (int)sizeof(float4) + BLOCK * (int)(sizeof(double) + 8);
}
template <int BLOCK>
struct MixedSmemT {
  float4 (*s)[BLOCK];
  double* lam_s;
  uint64_t* idx_s;
  GG_DEV float4 get(int slot) const { return s[slot][threadIdx.x]; }
  GG_DEV void set(int slot, float4 v) const { s[slot][threadIdx.x] = v; }
  GG_DEV float comp(int slot, int i) const {
    return reinterpret_cast<const float*>(&s[slot][threadIdx.x])[i];
  }
  GG_DEV double& lam() const { return lam_s[threadIdx.x]; }
  GG_DEV uint64_t& idx() const { return idx_s[threadIdx.x]; }
  // the column laid out in a CTA's dynamic shared memory
  GG_DEV static MixedSmemT at(void* smem) {
    auto* k = reinterpret_cast<float4(*)[BLOCK]>(smem);
    auto* lam = reinterpret_cast<double*>(reinterpret_cast<char*>(smem) +
                                          kMixedSlots * BLOCK * sizeof(float4));
    return {k, lam, reinterpret_cast<uint64_t*>(lam + BLOCK)};
  }
};
using MixedSmem = MixedSmemT<kTraceBlock>;

// Register part of a mixed-form ray.
struct MixedRegs {
  float vh[4];  // velocity, hi part
  double h;     // step size (controller state, FP64)
};

// Starts a ray: state from FP64, split into hi + lo.
template <class KS>
GG_DEV void mixed_load(const Ray& R, uint64_t idx, const KS& K, MixedRegs& S) {
  float xh[4], xl[4], vl[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    split(R.x[i], xh[i], xl[i]);
    split(R.v[i], S.vh[i], vl[i]);
  }
  K.set(kSlotXh, make_float4(xh[0], xh[1], xh[2], xh[3]));
  K.set(kSlotXl, make_float4(xl[0], xl[1], xl[2], xl[3]));
  K.set(kSlotVl, make_float4(vl[0], vl[1], vl[2], vl[3]));
  K.lam() = R.lam;
  K.idx() = idx;
  S.h = R.h;
}

// The ray's state in FP64 (hi + lo).
template <class KS>
GG_DEV Ray mixed_fp64(const KS& K, const MixedRegs& S) {
  const float4 xh = K.get(kSlotXh), xl = K.get(kSlotXl), vl = K.get(kSlotVl);
  Ray R;
  R.x[0] = (double)xh.x + (double)xl.x;
  R.x[1] = (double)xh.y + (double)xl.y;
  R.x[2] = (double)xh.z + (double)xl.z;
  R.x[3] = (double)xh.w + (double)xl.w;
  R.v[0] = (double)S.vh[0] + (double)vl.x;
  R.v[1] = (double)S.vh[1] + (double)vl.y;
  R.v[2] = (double)S.vh[2] + (double)vl.z;
  R.v[3] = (double)S.vh[3] + (double)vl.w;
  R.h = S.h;
  R.lam = K.lam();
  return R;
}

// Dormand-Prince coefficients as FP32 compile-time constants, so the unrolled
// stage sums fold them into the FMAs and drop the zero ones.
template <int S, int L>
struct DPc {
  static constexpr float abar = static_cast<float>(make_dp_table().Abar[S][L]);
  static constexpr float b = static_cast<float>(make_dp_table().B[S][L]);
};
template <int L>
struct DPe {
  static constexpr float e = static_cast<float>(make_dp_table().E[L]);
  static constexpr float ebar = static_cast<float>(make_dp_table().Ebar[L]);
};
template <int S>
struct DPa {
  static constexpr float a = static_cast<float>(make_dp_table().A[S]);
};

// ax += sum_l Abar[S][l] k_l, av += sum_l B[S][l] k_l over l < S.
template <int S, int L, class KS>
GG_DEV void stage_sums(const KS& K, float ax[4], float av[4]) {
  if constexpr (L < S) {
    constexpr float cb = DPc<S, L>::abar, cv = DPc<S, L>::b;
    if constexpr (cb != 0.0f || cv != 0.0f) {
      const float4 k4 = K.get(L);
      const float k[4] = {k4.x, k4.y, k4.z, k4.w};
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        if constexpr (cb != 0.0f) ax[i] = fmaf(cb, k[i], ax[i]);
        if constexpr (cv != 0.0f) av[i] = fmaf(cv, k[i], av[i]);
      }
    }
    stage_sums<S, L + 1>(K, ax, av);
  }
}

#if GG_MIXED_PAIRED
// The same sums with the paired FP32 fused multiply-add (two lanes of one
// instruction, each rounded as fmaf): the velocity sums over (t, r) and
// (theta, phi), and, for stage 6 whose four position increments are all
// used, the position sums too; stages 1-5 form only r and theta.  Same
// operations in the same order, so the same bits as stage_sums.
template <int S, int L, class KS>
GG_DEV void stage_sums2(const KS& K, float ax[4], float2& av01, float2& av23) {
  if constexpr (L < S) {
    constexpr float cb = DPc<S, L>::abar, cv = DPc<S, L>::b;
    if constexpr (cb != 0.0f || cv != 0.0f) {
      const float4 k4 = K.get(L);
      const float2 k01 = make_float2(k4.x, k4.y), k23 = make_float2(k4.z, k4.w);
      if constexpr (cb != 0.0f) {
        if constexpr (S == 6) {
          const float2 c2 = make_float2(cb, cb);
          const float2 a01 = __ffma2_rn(c2, k01, make_float2(ax[0], ax[1]));
          const float2 a23 = __ffma2_rn(c2, k23, make_float2(ax[2], ax[3]));
          ax[0] = a01.x;
          ax[1] = a01.y;
          ax[2] = a23.x;
          ax[3] = a23.y;
        } else {
          ax[1] = fmaf(cb, k4.y, ax[1]);
          ax[2] = fmaf(cb, k4.z, ax[2]);
        }
      }
      if constexpr (cv != 0.0f) {
        const float2 c2 = make_float2(cv, cv);
        av01 = __ffma2_rn(c2, k01, av01);
        av23 = __ffma2_rn(c2, k23, av23);
      }
    }
    stage_sums2<S, L + 1>(K, ax, av01, av23);
  }
}
#endif

// ex += sum_l Ebar_l k_l, ev += sum_l E_l k_l over the seven stages.
template <int L, class KS>
GG_DEV void error_sums(const KS& K, float ex[4], float ev[4]) {
  if constexpr (L < 7) {
    constexpr float eb = DPe<L>::ebar, e = DPe<L>::e;
    if constexpr (eb != 0.0f || e != 0.0f) {
      const float4 k4 = K.get(L);
      const float k[4] = {k4.x, k4.y, k4.z, k4.w};
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        if constexpr (eb != 0.0f) ex[i] = fmaf(eb, k[i], ex[i]);
        if constexpr (e != 0.0f) ev[i] = fmaf(e, k[i], ev[i]);
      }
    }
    error_sums<L + 1>(K, ex, ev);
  }
}

// The same sums in FP64 over the FP32 stage derivatives (each product and
// sum carries the FP64 rounding only), the coefficients in FP64.
template <int L, class KS>
GG_DEV void error_sums64(const KS& K, double ex[4], double ev[4]) {
  if constexpr (L < 7) {
    constexpr double eb = make_dp_table().Ebar[L], e = make_dp_table().E[L];
    if constexpr (eb != 0.0 || e != 0.0) {
      const float4 k4 = K.get(L);
      const double k[4] = {(double)k4.x, (double)k4.y, (double)k4.z, (double)k4.w};
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        if constexpr (eb != 0.0) ex[i] = fma(eb, k[i], ex[i]);
        if constexpr (e != 0.0) ev[i] = fma(e, k[i], ev[i]);
      }
    }
    error_sums64<L + 1>(K, ex, ev);
  }
}

// Stage S's r, theta and velocity as increments over the state's hi part:
// x_S = x + h a_S v + h^2 sum Abar k, v_S = v + h sum B k.  Stage 6 is the
// 5th-order solution: its four position and velocity increments are the
// step's dx, dv (slots 7, 8).
template <int S, class KS>
GG_DEV void mixed_stage(float r0, float th0, const MixedRegs& st, const KS& K, float hf,
                        float hh, float& pr, float& pth, float pw[4]) {
  float ax[4] = {0.0f, 0.0f, 0.0f, 0.0f}, av[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#if GG_MIXED_PAIRED
  float2 av01 = make_float2(0.0f, 0.0f), av23 = make_float2(0.0f, 0.0f);
  stage_sums2<S, 0>(K, ax, av01, av23);
  if constexpr (S != 6) {  // the stage velocity, paired: v + h sum B k
    const float2 h2 = make_float2(hf, hf);
    const float2 w01 = __ffma2_rn(h2, av01, make_float2(st.vh[0], st.vh[1]));
    const float2 w23 = __ffma2_rn(h2, av23, make_float2(st.vh[2], st.vh[3]));
    pw[0] = w01.x;
    pw[1] = w01.y;
    pw[2] = w23.x;
    pw[3] = w23.y;
    const float ha = hf * DPa<S>::a;
    pr = r0 + fmaf(hh, ax[1], ha * st.vh[1]);
    pth = th0 + fmaf(hh, ax[2], ha * st.vh[2]);
    return;
  }
  av[0] = av01.x;
  av[1] = av01.y;
  av[2] = av23.x;
  av[3] = av23.y;
#else
  stage_sums<S, 0>(K, ax, av);
#endif
  const float ha = hf * DPa<S>::a;
  float dx[4], dv[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    dx[i] = fmaf(hh, ax[i], ha * st.vh[i]);
    if constexpr (S == 6) {  // the step's increments: v_new = v + dv exactly as stored
      dv[i] = hf * av[i];
      pw[i] = st.vh[i] + dv[i];
    } else {
      pw[i] = fmaf(hf, av[i], st.vh[i]);
    }
  }
  pr = r0 + dx[1];
  pth = th0 + dx[2];
  if constexpr (S == 6) {
    K.set(kSlotDx, make_float4(dx[0], dx[1], dx[2], dx[3]));
    K.set(kSlotDv, make_float4(dv[0], dv[1], dv[2], dv[3]));
  }
}

// kerr_geometry in FP32 with the render's constant products (2M, a^2,
// 2Ma, ... in DevParams) taken as given rather than rebuilt per evaluation:
// the same symbols, a dozen fewer multiplies per right-hand side.
GG_DEV KerrGeo<float> kerr_geometry32(const DevParams& P, float r, float s, float c) {
  KerrGeo<float> G;
  const float a2 = P.a2_f;
  const float r2 = r * r, s2 = s * s, c2 = c * c, sc = s * c;
  const float sig = fmaf(a2, c2, r2);
  const float del = fmaf(r - P.m2_f, r, a2);
  const float rho = r2 + a2;
  const float sd = sig * del;
  const float R = rcp(sd * s2);
  const float iSD = s2 * R;   // 1 / (Sigma Delta)
  const float iS = del * iSD;  // 1 / Sigma
  const float iD = sig * iSD;  // 1 / Delta
  const float is2 = sd * R;    // 1 / sin^2
  const float iS2 = iS * iS;
  const float sm2r = fmaf(a2, c2, -r2);  // Sigma - 2 r^2
  const float sm2r_iS2 = sm2r * iS2;
  const float rsc_iS2 = r * (sc * iS2);
  G.dtt_r = P.m2_f * sm2r_iS2;
  G.dtt_th = P.m4a2_f * rsc_iS2;
  G.drr_r = 2.0f * fmaf(a2, fmaf(r, s2, P.mass_f * c2), -P.mass_f * r2) * (iD * iD);
  G.drr_th = P.mm2a2_f * sc * iD;
  G.dthth_r = 2.0f * r;
  G.dthth_th = P.mm2a2_f * sc;
  G.dphph_r = fmaf(2.0f * r, s2, P.m2a2_f * (s2 * s2) * sm2r_iS2);
  G.dphph_th = fmaf(2.0f * rho, sc, P.m4a2_f * rsc_iS2 * s2 * (sig + rho));
  G.dtph_r = -P.m2a_f * s2 * sm2r_iS2;
  G.dtph_th = -P.m4a_f * rsc_iS2 * rho;
  const float big_a = fmaf(rho, rho, -a2 * del * s2);
  G.gtt = -big_a * iSD;
  G.gtph = -P.m2a_f * r * iSD;
  G.gphph = fmaf(-a2, s2, del) * iSD * is2;
  G.hrr = -0.5f * del * iS;
  G.hthth = -0.5f * iS;
  return G;
}

// kerr_contract in FP32, the r and theta rows reusing the t and phi rows'
// sums: with A = G_tt vt + G_tph vph and B = G_tph vt + G_phph vph (per row),
// G_tt vt^2 + 2 G_tph vt vph + G_phph vph^2 = vt A + vph B.  The same symbols,
// four fewer operations per right-hand side.
GG_DEV void kerr_contract32(const KerrGeo<float>& G, const float v[4], float acc[4]) {
  const float vt = v[0], vr = v[1], vth = v[2], vph = v[3];
  const float Ar = fmaf(G.dtph_r, vph, G.dtt_r * vt);
  const float Br = fmaf(G.dphph_r, vph, G.dtph_r * vt);
  const float Ath = fmaf(G.dtph_th, vph, G.dtt_th * vt);
  const float Bth = fmaf(G.dphph_th, vph, G.dtph_th * vt);
  const float Et = fmaf(vth, Ath, vr * Ar);
  const float Ep = fmaf(vth, Bth, vr * Br);
  acc[0] = -fmaf(G.gtph, Ep, G.gtt * Et);
  acc[3] = -fmaf(G.gphph, Ep, G.gtph * Et);
  // r row: drr_r vr^2 + 2 drr_th vr vth - dthth_r vth^2 - (vt Ar + vph Br)
  float w = vr * fmaf(G.drr_r, vr, (G.drr_th + G.drr_th) * vth);
  w = fmaf(-G.dthth_r, vth * vth, w);
  w = fmaf(-vt, Ar, w);
  w = fmaf(-vph, Br, w);
  acc[1] = G.hrr * w;
  // theta row: dthth_th vth^2 + 2 dthth_r vr vth - drr_th vr^2 - (vt Ath + vph Bth)
  float u = vth * fmaf(G.dthth_th, vth, (G.dthth_r + G.dthth_r) * vr);
  u = fmaf(-G.drr_th, vr * vr, u);
  u = fmaf(-vt, Ath, u);
  u = fmaf(-vph, Bth, u);
  acc[2] = G.hthth * u;
}

template <int METRIC>
struct Geometry32;

template <>
struct Geometry32<kMetricKerr> {
  KerrGeo<float> g;
  GG_DEV void at(const DevParams& P, float r, float th) {
    float s, c;
    sincos_polar(th, &s, &c);
    g = kerr_geometry32(P, fmaxf(r, 1e-10f), s, c);
  }
  GG_DEV void accel(const float v[4], float a[4]) const { kerr_contract32(g, v, a); }
};

template <>
struct Geometry32<kMetricSchwarzschild> {
  SchwGeoT<float> g;
  GG_DEV void at(const DevParams& P, float r, float th) {
    float s, c;
    sincos_polar(th, &s, &c);
    g = schw_geometry<float>(P.rs_f, fmaxf(r, 1e-10f), s, c);
  }
  GG_DEV void accel(const float v[4], float a[4]) const { schw_contract<float>(g, v, a); }
};

// x^(1/5) for x in (1, 1e30], larger x taken as 1e30: on acceptance
// x = tol/err > 1, and a root above 1e6 only matters through the max_step
// clamp.  Same seed-and-Newton scheme as fifth_root, without its pow branch.
GG_DEV double fifth_root_accept(double x) {
  x = fmin(x, 1e30);
  double z = (double)__powf((float)x, -0.2f);
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const double z2 = z * z;
    z = z * (1.2 - 0.2 * x * (z2 * z2 * z));
  }
  const double z2 = z * z;
  return x * (z2 * z2);
}

// (8 / s2)^(1/10) for s2 in (0, 8): the step factor (tol / err)^(1/5) of an
// accepted attempt with err = sqrt(s2 / 8), tol = 1, without forming err or
// the quotient.  s2 below 8e-60 is taken as 8e-60 (a factor of 1e6, as
// fifth_root_accept's clamp at 1e30).  Newton on w = y^(-1/10), y = s2 / 8:
// w <- w (1.1 - 0.1 y w^10), two iterations from the FP32 power.  Below
// s2 = 8e-30 the float seed would underflow, so y is scaled by 1e30 and the
// result by 1e3.  Measured against the exact root (w^10 s2 / 8 in rational
// arithmetic) over s2 from 1e-70 to 8: within 3.8e-16, about 2 ulp; a third
// iteration for small norms changed nothing and cost the 2,048-scene batch 3 %.
GG_DEV double root10_8_over(double s2) {
  s2 = fmax(s2, 8e-60);
  const bool tiny = s2 < 8e-30;
  const double y = tiny ? s2 * 1.25e29 : s2 * 0.125;
  double w = (double)__powf((float)y, -0.1f);
  const double ty = 0.1 * y;
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const double w2 = w * w, w4 = w2 * w2, w5 = w4 * w;
    w = w * fma(-ty, w5 * w5, 1.1);
  }
  return tiny ? w * 1e3 : w;
}

// The escape test of the reference's step (geodesic.rs:195-197) on the
// float-pair radius.
template <class KS>
GG_DEV bool beyond_max_radius(const DevParams& P, const KS& K) {
  return ff_minus(K.comp(kSlotXh, 1), K.comp(kSlotXl, 1), P.max_radius_hi, P.max_radius_lo) >
         0.0f;
}

// One mixed-precision attempt of the full Dormand-Prince step.  Control flow
// is attempt_dp45_fp64's: escape test, invalid-stage halving, acceptance test
// and step-size law (FP64).  On acceptance the state is NOT advanced: the
// increments are in slots 7 and 8 and hf is the step taken, so the caller
// can test the step for crossings against the pre-step state first
// (mixed_advance applies it).  The horizon test never fires here: the FP64
// band starts 0.5 M outside the horizon and its buffer.  Invalid stages are
// judged on r and theta, the coordinates the stages form.
template <int METRIC, class KS>
GG_DEV int attempt_dp45_mixed(const DevParams& P, MixedRegs& S, const KS& K,
                              bool& k1_valid, bool& k7_pending, bool& accepted, float& hf) {
  accepted = false;
  if (beyond_max_radius(P, K)) return kEscaped;
  if (k7_pending) {
    K.set(0, K.get(6));
    k7_pending = false;
  }
  hf = (float)S.h;
  const float hh = hf * hf;
  const float r0 = K.comp(kSlotXh, 1), th0 = K.comp(kSlotXh, 2);
  const int s_first = __any_sync(__activemask(), !k1_valid) ? 0 : 1;
  // One stage: its inputs, the validity test of its position (false: the
  // attempt ends with h halved), the right-hand side, k_s stored.
  auto stage = [&](int s) -> bool {
    float pr, pth, pw[4];
    switch (s) {
      case 0:
        pr = r0;
        pth = th0;
#pragma unroll
        for (int i = 0; i < 4; ++i) pw[i] = S.vh[i];
        break;
      case 1: mixed_stage<1>(r0, th0, S, K, hf, hh, pr, pth, pw); break;
      case 2: mixed_stage<2>(r0, th0, S, K, hf, hh, pr, pth, pw); break;
      case 3: mixed_stage<3>(r0, th0, S, K, hf, hh, pr, pth, pw); break;
      case 4: mixed_stage<4>(r0, th0, S, K, hf, hh, pr, pth, pw); break;
      case 5: mixed_stage<5>(r0, th0, S, K, hf, hh, pr, pth, pw); break;
      default: mixed_stage<6>(r0, th0, S, K, hf, hh, pr, pth, pw); break;
    }
    if (s > 0 && !(isfinite(pr) && isfinite(pth) && pr > 0.0f)) return false;
    Geometry32<METRIC> G;
    G.at(P, pr, pth);
    float a[4];
    G.accel(pw, a);
    // a lane whose k1 is valid keeps it when its warp recomputes stage 0
    // for a refilled lane: k7 was evaluated at the stage position formed as
    // an FP32 increment, which differs in the last bits from the
    // compensated state, so overwriting it would make a ray's result depend
    // on which rays share its warp
    if (s > 0 || !k1_valid) K.set(s, make_float4(a[0], a[1], a[2], a[3]));
    return true;
  };
#if GG_MIXED_STAGE_UNROLL
  if (s_first == 0) stage(0);
#pragma unroll
  for (int s = 1; s < 7; ++s) {
    if (!stage(s)) {
      S.h = S.h * 0.5;
      return kContinue;
    }
  }
#else
#pragma unroll 1
  for (int s = s_first; s < 7; ++s) {
    if (!stage(s)) {
      S.h = S.h * 0.5;
      return kContinue;
    }
  }
#endif
  const float4 dx4 = K.get(kSlotDx), dv4 = K.get(kSlotDv), xh4 = K.get(kSlotXh);
  const float dx[4] = {dx4.x, dx4.y, dx4.z, dx4.w}, dv[4] = {dv4.x, dv4.y, dv4.z, dv4.w};
  const float xh[4] = {xh4.x, xh4.y, xh4.z, xh4.w};
  double err, tol;
#if GG_MIXED_ERR_FP64
  // The embedded error estimate in FP64: the sums over the FP32 stage
  // derivatives (exact in FP64 up to the final rounding), scaled and reduced
  // in FP64; the per-component scale atol + rtol max(|y|, |y_new|) is a
  // weight and stays FP32.
  double ex[4] = {0.0, 0.0, 0.0, 0.0}, ev[4] = {0.0, 0.0, 0.0, 0.0};
  error_sums64<0>(K, ex, ev);
  const double hd = (double)hf, hhd = hd * hd;  // both exact
  double s2 = 0.0;
  if (P.rtol > 0.0) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const float xs = fmaf(P.rtol_f, fmaxf(fabsf(xh[i]), fabsf(xh[i] + dx[i])), P.atol_f);
      const float vs = fmaf(P.rtol_f, fmaxf(fabsf(S.vh[i]), fabsf(S.vh[i] + dv[i])), P.atol_f);
      const double qx = (hhd * ex[i]) * (double)__fdividef(1.0f, xs);
      const double qv = (hd * ev[i]) * (double)__fdividef(1.0f, vs);
      s2 = fma(qx, qx, fma(qv, qv, s2));
    }
#if GG_MIXED_ROOT10
    // err = sqrt(s2 / 8) < tol = 1 is s2 < 8; the step laws in s2 directly
    if (s2 < 8.0 || S.h <= P.min_step) {
      accepted = true;
      if (s2 > 0.0) {
        double hn = S.h * 0.9 * root10_8_over(s2);
        hn = hn < P.min_step ? P.min_step : (hn > P.max_step ? P.max_step : hn);
        S.h = hn;
      }
    } else {
      S.h = fmax(S.h * 0.9 * sqrt(sqrt(sqrt(8.0 / s2))), P.min_step);
    }
    return kContinue;
#endif
    err = sqrt(s2 * 0.125);
    tol = 1.0;
  } else {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const double ax = hhd * ex[i], av = hd * ev[i];
      s2 = fma(ax, ax, fma(av, av, s2));
    }
    err = sqrt(s2);
    tol = P.tolerance;
  }
#else
  float ex[4] = {0.0f, 0.0f, 0.0f, 0.0f}, ev[4] = {0.0f, 0.0f, 0.0f, 0.0f};
  error_sums<0>(K, ex, ev);
  float s2 = 0.0f;
  if (P.rtol > 0.0) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const float xs = fmaf(P.rtol_f, fmaxf(fabsf(xh[i]), fabsf(xh[i] + dx[i])), P.atol_f);
      const float vs = fmaf(P.rtol_f, fmaxf(fabsf(S.vh[i]), fabsf(S.vh[i] + dv[i])), P.atol_f);
      const float qx = __fdividef(hh * ex[i], xs);
      const float qv = __fdividef(hf * ev[i], vs);
      s2 = fmaf(qx, qx, fmaf(qv, qv, s2));
    }
    err = sqrt((double)s2 * 0.125);
    tol = 1.0;
  } else {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const float ax = hh * ex[i], av = hf * ev[i];
      s2 = fmaf(ax, ax, fmaf(av, av, s2));
    }
    err = sqrt((double)s2);
    tol = P.tolerance;
  }
#endif
  if (err < tol || S.h <= P.min_step) {
    accepted = true;
    if (err > 0.0) {
      double hn = S.h * 0.9 * fifth_root_accept(tol / err);
      hn = hn < P.min_step ? P.min_step : (hn > P.max_step ? P.max_step : hn);
      S.h = hn;
    }
  } else {
    S.h = fmax(S.h * 0.9 * sqrt(sqrt(tol / err)), P.min_step);
  }
  return kContinue;
}

// Applies an accepted attempt's increments (compensated) and wraps phi into
// [0, 2 pi); k7 becomes the next attempt's k1.
template <class KS>
GG_DEV void mixed_advance(MixedRegs& S, const KS& K, float hf, bool& k1_valid,
                          bool& k7_pending) {
  const float4 dx4 = K.get(kSlotDx), dv4 = K.get(kSlotDv);
  const float4 xh4 = K.get(kSlotXh), xl4 = K.get(kSlotXl), vl4 = K.get(kSlotVl);
  float xh[4] = {xh4.x, xh4.y, xh4.z, xh4.w}, xl[4] = {xl4.x, xl4.y, xl4.z, xl4.w};
  float vl[4] = {vl4.x, vl4.y, vl4.z, vl4.w};
  const float dx[4] = {dx4.x, dx4.y, dx4.z, dx4.w}, dv[4] = {dv4.x, dv4.y, dv4.z, dv4.w};
#if GG_MIXED_PAIRED
#pragma unroll
  for (int j = 0; j < 4; j += 2) {
    float2 h = make_float2(xh[j], xh[j + 1]), l = make_float2(xl[j], xl[j + 1]);
    ff_add2(h, l, make_float2(dx[j], dx[j + 1]));
    xh[j] = h.x;
    xh[j + 1] = h.y;
    xl[j] = l.x;
    xl[j + 1] = l.y;
    float2 vh2 = make_float2(S.vh[j], S.vh[j + 1]), vl2 = make_float2(vl[j], vl[j + 1]);
    ff_add2(vh2, vl2, make_float2(dv[j], dv[j + 1]));
    S.vh[j] = vh2.x;
    S.vh[j + 1] = vh2.y;
    vl[j] = vl2.x;
    vl[j + 1] = vl2.y;
  }
#else
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    ff_add(xh[i], xl[i], dx[i]);
    ff_add(S.vh[i], vl[i], dv[i]);
  }
#endif
  if (xh[3] >= kTwoPiHi) {
    ff_add(xh[3], xl[3], -kTwoPiHi);
    ff_add(xh[3], xl[3], -kTwoPiLo);
  } else if (xh[3] < 0.0f) {
    ff_add(xh[3], xl[3], kTwoPiHi);
    ff_add(xh[3], xl[3], kTwoPiLo);
  }
  K.set(kSlotXh, make_float4(xh[0], xh[1], xh[2], xh[3]));
  K.set(kSlotXl, make_float4(xl[0], xl[1], xl[2], xl[3]));
  K.set(kSlotVl, make_float4(vl[0], vl[1], vl[2], vl[3]));
  K.lam() = K.lam() + (double)hf;
  k1_valid = true;
  k7_pending = true;
}

}  // namespace gg
