// gg_adjoint.cu -- the differentiable render: forward pass with checkpoints
// and the hand-written adjoint (reverse-mode) pass.
//
// Image: Kerr, thin disk, one sample per pixel, full Dormand-Prince stepper
// in FP64.  Each pixel's linear colour is a function of five parameters:
// spin a, camera inclination and distance (the inclined camera of
// gg_camera_inclined), disk inner radius r_in and emissivity index q.  Disk
// pixels carry I = g^4 (r_in / r_c)^q through the disk colour; sky and
// horizon pixels are piecewise constant in the parameters (zero gradient;
// their jumps across class or cell boundaries are not differentiated).
//
// Forward (gg_forward_ckpt): the FP64 trace kernel's checkpointing variant
// (trace_fp64_kernel<Kerr, thin disk, full Dormand-Prince, ..., CKPT> in
// gg_trace.cu), which also stores each ray's state (x, v, next h) at the start
// and after every kCkptEvery-th accepted step, and its DiffRay.
//
// Backward (diff_backward_kernel), per disk ray, given dL/d(colour):
//   1. the crossing step (the last accepted step) again in forward-mode dual
//      numbers over its start state (8) and the spin: stages, continuous
//      extension, the root s* (one Newton correction in dual arithmetic gives
//      ds*/dp by the implicit function theorem), the crossing state, the
//      redshift and I -- so dL/d(start state), dL/da, dL/dr_in, dL/dq and
//      dL/d(observer normalisation) in one pass;
//   2. every earlier step in reverse, segment by segment: the segment is
//      replayed from its checkpoint (the controller is deterministic, so the
//      replay takes the same steps), then the adjoint goes back through each
//      step's Dormand-Prince stages (vector-Jacobian products of each
//      stage's Kerr right-hand side in r, theta, the stage velocity and the
//      spin, by a hand-written reverse pass, gg_vjp.cuh), with theta
//      reflections at the poles reversing its adjoint;
//   3. the camera: the initial state and the observer normalisation as
//      3-direction duals in (a, inclination, r_cam), contracted with the
//      adjoint of the initial state.
// The step sizes are held fixed (the adjoint of the discrete map with the
// forward's accepted steps; their own dependence on the parameters moves the
// solution by the truncation error only).
#include <cuda_runtime.h>

#include <cstdint>

#include "gg_device.cuh"
#include "gg_dual.cuh"
#include "gg_vjp.cuh"
#include "gg_launch.h"
#include "gg_trace_common.cuh"

// Build knobs of the backward (tuning builds compare them).  GG_ADJ_HAND_VJP:
// each stage's vector-Jacobian product by the hand-written reverse pass
// (kerr_rhs_vjp_hand) instead of dual numbers.  GG_ADJ_STORE_K: the replay
// keeps each accepted step's stage derivatives for the step's product instead
// of evaluating them again.  GG_ADJ_MIN_BLOCKS: the CTAs per SM the backward's
// registers are budgeted for (1 leaves the compiler's own choice).  Measured
// on the 512^2 gradient (backward ms): dual numbers 11.2, dual with kept stages
// 9.9, hand-written 8.5, hand-written with kept stages 7.9 (the default; the
// forward takes 8.8); the gradients agree to 1e-15.  The same at 3 CTAs per SM
// (168 registers, twice the spill code): 9.0.
#ifndef GG_ADJ_HAND_VJP
#define GG_ADJ_HAND_VJP 1
#endif
#ifndef GG_ADJ_STORE_K
#define GG_ADJ_STORE_K 1
#endif
#ifndef GG_ADJ_MIN_BLOCKS
#define GG_ADJ_MIN_BLOCKS 1
#endif

namespace gg {

namespace {

// a^mu of one Kerr right-hand side in dual arithmetic (no r clamp: valid
// stages have r > 0).
template <int N>
GG_DEV void kerr_rhs_dual(double M, const Dual<N>& a, const Dual<N>& r, const Dual<N>& th,
                          const Dual<N> w[4], Dual<N> acc[4]) {
  Dual<N> s, c;
  sincos(th, &s, &c);
  const KerrGeo<Dual<N>> G = kerr_geometry<Dual<N>>(Dual<N>(M), a, r, s, c);
  kerr_contract<Dual<N>>(G, w, acc);
}

// g of a Keplerian emitter at the equator (redshift_factor at theta = pi/2)
// without the observer normalisation (divide by sqrt(-g_tt) at the camera).
template <class T>
GG_DEV T redshift_eq(double M, const T& a, const T& r, const T v[4]) {
  const T gtt = -(1.0 - 2.0 * M / r);
  const T gtph = -2.0 * M * a / r;
  const T gphph = r * r + a * a + 2.0 * M * a * a / r;
  const T p_t = gtt * v[0] + gtph * v[3];
  const double sm = ::sqrt(M);
  const T omega = sm / (r * sqrt(r) + a * sm);
  const T denom = -(gtt + 2.0 * gtph * omega + gphph * omega * omega);
  const T u_t = 1.0 / sqrt(denom);
  const T u_p = omega * u_t;
  const T p_phi = gtph * v[0] + gphph * v[3];
  const T e_emit = -(p_t * u_t + p_phi * u_p);
  return -p_t / e_emit;
}

// ---- backward -----------------------------------------------------------------
// Vector-Jacobian product through one accepted full Dormand-Prince step
// (Nystrom form, attempt_dp45_fp64): (lx, lv) is dL/d(x_new, v_new) on entry
// and dL/d(x, v) on return; dL/da is accumulated into *ga.
// kst: the step's stage derivatives k_1..k_6 as the forward took them, or
// null to evaluate them again here.
GG_DEV void dp45_vjp(const DevParams& P, const double x[4], const double v[4], double h,
                     const double (*kst)[4], double lx[4], double lv[4], double* ga) {
  double k[6][4], pr[6], pth[6], pw[6][4];
  const double hh = h * h;
  for (int s = 0; s < 6; ++s) {
    double px[4], w[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      px[i] = fma(h * kDP.A[s], v[i], x[i]);
      w[i] = v[i];
    }
    for (int l = 0; l < s; ++l)
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        px[i] = fma(hh * kDP.Abar[s][l], k[l][i], px[i]);
        w[i] = fma(h * kDP.B[s][l], k[l][i], w[i]);
      }
    if (kst) {
#pragma unroll
      for (int i = 0; i < 4; ++i) k[s][i] = kst[s][i];
    } else {
      Geometry<kMetricKerr> G;
      G.at(P, px[1], px[2]);
      G.accel(w, k[s]);
    }
    pr[s] = px[1];
    pth[s] = px[2];
#pragma unroll
    for (int i = 0; i < 4; ++i) pw[s][i] = w[i];
  }
  double kb[6][4];
  for (int l = 0; l < 6; ++l)
#pragma unroll
    for (int i = 0; i < 4; ++i) kb[l][i] = 0.0;
  // outputs: x_new = x + h v + h^2 sum Abar[6][l] k_l, v_new = v + h sum B[6][l] k_l
  double xbar[4], vbar[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    xbar[i] = lx[i];
    vbar[i] = lv[i] + h * lx[i];
  }
  for (int l = 0; l < 6; ++l)
#pragma unroll
    for (int i = 0; i < 4; ++i) kb[l][i] += hh * kDP.Abar[6][l] * lx[i] + h * kDP.B[6][l] * lv[i];
  for (int s = 5; s >= 0; --s) {
    // k_s = f(r_s, theta_s, w_s; a), back through its Jacobian
    double Xr = 0.0, Xth = 0.0, W[4] = {0.0, 0.0, 0.0, 0.0};
#if GG_ADJ_HAND_VJP
    kerr_rhs_vjp_hand(P.mass, P.spin, pr[s], pth[s], pw[s], kb[s], &Xr, &Xth, W, ga);
#else
    kerr_rhs_vjp_dual(P.mass, P.spin, pr[s], pth[s], pw[s], kb[s], &Xr, &Xth, W, ga);
#endif
    // x_s = x + h A_s v + h^2 sum_{l<s} Abar k_l ; w_s = v + h sum_{l<s} B k_l
    xbar[1] += Xr;
    xbar[2] += Xth;
    vbar[1] += h * kDP.A[s] * Xr;
    vbar[2] += h * kDP.A[s] * Xth;
#pragma unroll
    for (int m = 0; m < 4; ++m) vbar[m] += W[m];
    for (int l = 0; l < s; ++l) {
      const double cb = hh * kDP.Abar[s][l], cv = h * kDP.B[s][l];
      kb[l][1] += cb * Xr;
      kb[l][2] += cb * Xth;
#pragma unroll
      for (int m = 0; m < 4; ++m) kb[l][m] += cv * W[m];
    }
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    lx[i] = xbar[i];
    lv[i] = vbar[i];
  }
}

// dL/d(start state of the crossing step) and the parameter terms of the
// crossing: the step, its continuous extension and root, the redshift and the
// disk colour in 9-direction duals (8 state components, spin).  dl: dL/d rgb.
// Returns false when the step does not reach the disk (no contribution).
GG_DEV bool crossing_vjp(const DevParams& P, const double xb[4], const double vb[4], double h,
                         const double dl[3], double lam[8], double* ga, double* g_rin,
                         double* g_q, double* g_sobs) {
  using D9 = Dual<9>;
  D9 x[4], v[4], k[7][4], xa[4], va[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    x[i] = D9::var(xb[i], i);
    v[i] = D9::var(vb[i], 4 + i);
  }
  const D9 a = D9::var(P.spin, 8);
  const double hh = h * h;
  for (int s = 0; s < 7; ++s) {
    D9 px[4], w[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      px[i] = x[i] + (h * kDP.A[s]) * v[i];
      w[i] = v[i];
    }
    for (int l = 0; l < s; ++l)
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        px[i] = px[i] + (hh * kDP.Abar[s][l]) * k[l][i];
        w[i] = w[i] + (h * kDP.B[s][l]) * k[l][i];
      }
    kerr_rhs_dual<9>(P.mass, a, px[1], px[2], w, k[s]);
    if (s == 6) {
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        xa[i] = px[i];
        va[i] = w[i];
      }
    }
  }
  // continuous extension coefficients of the 8 components
  D9 y0[8], r2[8], r3[8], r4[8], r5[8];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    D9 sx(0.0), sv(0.0);
    for (int l = 0; l < 7; ++l) {
      sx = sx + kDP.Dbar[l] * k[l][i];
      sv = sv + kDP.D[l] * k[l][i];
    }
    y0[i] = x[i];
    r2[i] = xa[i] - x[i];
    r3[i] = h * v[i] - r2[i];
    r4[i] = r2[i] - h * va[i] - r3[i];
    r5[i] = hh * sx;
    y0[4 + i] = v[i];
    r2[4 + i] = va[i] - v[i];
    r3[4 + i] = h * k[0][i] - r2[4 + i];
    r4[4 + i] = r2[4 + i] - h * k[6][i] - r3[4 + i];
    r5[4 + i] = h * sv;
  }
  // the root on values (safeguarded Newton), then one Newton step in duals
  StepSpan sp;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    sp.xb[i] = xb[i];
    sp.vb[i] = vb[i];
    sp.xa[i] = xa[i].v;
    sp.va[i] = va[i].v;
  }
  for (int l = 0; l < 7; ++l)
#pragma unroll
    for (int i = 0; i < 4; ++i) sp.k[l][i] = k[l][i].v;
  sp.h = h;
  double cval[8];
  const double s0 = dense_crossing(sp, 2, kHalfPi, cval);
  auto poly = [&](int c, const D9& s) {
    const D9 t = 1.0 - s;
    return y0[c] + s * (r2[c] + t * (r3[c] + s * (r4[c] + t * r5[c])));
  };
  const D9 sd0(s0);
  const D9 f = poly(2, sd0) - kHalfPi;
  const double t0 = 1.0 - s0;
  const double fp = r2[2].v + (1.0 - 2.0 * s0) * r3[2].v + s0 * (2.0 - 3.0 * s0) * r4[2].v +
                    2.0 * s0 * t0 * (1.0 - 2.0 * s0) * r5[2].v;
  const D9 sd = sd0 - f / fp;
  const D9 rc = poly(1, sd);
  double rcv = rc.v;
  {
    double cn[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) cn[c] = cval[c];
    normalize_coords(cn);
    rcv = cn[1];
  }
  if (!(rcv >= P.r_inner && rcv <= P.r_outer)) return false;
  D9 vc[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) vc[i] = poly(4 + i, sd);
  // g (observer normalisation s_obs factored out), I = g^4 (r_in / r_c)^q
  const D9 g0 = redshift_eq<D9>(P.mass, a, rc, vc);
  const D9 g = g0 / P.sqrt_neg_gtt_obs;
  const D9 g2 = g * g;
  const D9 I = (g2 * g2) * pow(P.r_inner / rc, P.emissivity_index);
  // dL/dI through the disk colour (x^0.5, x^1.2, x^2.5), x = I / (1 + I)
  const double xv = I.v / (1.0 + I.v);
  const double dx = 1.0 / ((1.0 + I.v) * (1.0 + I.v));
  const double dLdI = dx * (dl[0] * 0.5 * ::pow(xv, -0.5) + dl[1] * 1.2 * ::pow(xv, 0.2) +
                            dl[2] * 2.5 * ::pow(xv, 1.5));
#pragma unroll
  for (int j = 0; j < 8; ++j) lam[j] = dLdI * I.d[j];
  *ga += dLdI * I.d[8];
  *g_rin += dLdI * I.v * P.emissivity_index / P.r_inner;
  *g_q += dLdI * I.v * ::log(P.r_inner / rc.v);
  *g_sobs += dLdI * (-4.0 * I.v / P.sqrt_neg_gtt_obs);
  return true;
}

// The initial state and the observer normalisation as functions of (a,
// inclination, r_cam) for image-plane point (u, v): the inclined camera
// (look_at = -r_hat, up = +z) and GeodesicRay::from_camera, in duals.
GG_DEV void camera_dual(const DevParams& P, double u, double v, Dual<3> y0[8], Dual<3>* sobs) {
  using D3 = Dual<3>;
  const D3 a = D3::var(P.spin, 0), th = D3::var(P.cam_pos[2], 1), r = D3::var(P.cam_pos[1], 2);
  D3 st, ct;
  sincos(th, &st, &ct);
  const D3 fwd[3] = {-st, D3(0.0), -ct};
  // right = normalize(fwd x up), up' = normalize(right x fwd), up = +z
  D3 right[3] = {fwd[1], -fwd[0], D3(0.0)};
  const D3 rn = sqrt(right[0] * right[0] + right[1] * right[1]);
  right[0] = right[0] / rn;
  right[1] = right[1] / rn;
  D3 up2[3] = {right[1] * fwd[2] - right[2] * fwd[1], right[2] * fwd[0] - right[0] * fwd[2],
               right[0] * fwd[1] - right[1] * fwd[0]};
  const D3 un = sqrt(up2[0] * up2[0] + up2[1] * up2[1] + up2[2] * up2[2]);
#pragma unroll
  for (int i = 0; i < 3; ++i) up2[i] = up2[i] / un;
  D3 d[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) d[i] = fwd[i] + (u * P.half_w) * right[i] + (v * P.half_h) * up2[i];
  const D3 dn = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  // local frame at phi = 0: r_hat = (st, 0, ct), theta_hat = (ct, 0, -st), phi_hat = (0, 1, 0)
  const D3 n_r = (d[0] * st + d[2] * ct) / dn;
  const D3 n_t = (d[0] * ct - d[2] * st) / dn;
  const D3 n_p = d[1] / dn;
  // Kerr metric at the camera (kerr.rs:61-94, no g_tphi, as the reference)
  const double M = P.mass;
  const D3 sig = r * r + a * a * ct * ct;
  const D3 del = r * r - 2.0 * M * r + a * a;
  const D3 gtt = -(1.0 - 2.0 * M * r / sig);
  const D3 grr = sig / del;
  const D3 gthth = sig;
  const D3 gphph = (r * r + a * a + 2.0 * M * a * a * r * st * st / sig) * st * st;
  const D3 kr = n_r / sqrt(grr), kth = n_t / sqrt(gthth), kph = n_p / sqrt(gphph);
  const D3 sns = grr * kr * kr + gthth * kth * kth + gphph * kph * kph;
  y0[0] = D3(P.cam_pos[0]);
  y0[1] = r;
  y0[2] = th;
  y0[3] = D3(P.cam_pos[3]);
  y0[4] = sqrt(-sns / gtt);
  y0[5] = kr;
  y0[6] = kth;
  y0[7] = kph;
  *sobs = sqrt(-gtt);
}

// Replays one segment of accepted steps from a checkpoint, recording each
// step's start state, size and whether its end was reflected at a pole, and
// (Kst non-null) its stage derivatives k_1..k_6.
GG_DEV void replay(const DevParams& P, const Ckpt& c0, uint32_t steps, double S[][8], double* H,
                   double (*Kst)[6][4], uint32_t* refl) {
  double kl[7][4];
  const KStoreLocal K{kl};
  Ray R;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    R.x[i] = c0.x[i];
    R.v[i] = c0.v[i];
  }
  R.h = c0.h;
  R.lam = 0.0;
  bool k1v = false, k7p = false;
  *refl = 0u;
  for (uint32_t j = 0; j < steps; ++j) {
    for (uint32_t guard = 0; guard < 100000u; ++guard) {
      double xb[4], vb[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        xb[i] = R.x[i];
        vb[i] = R.v[i];
      }
      bool acc;
      double h_used = 0.0;
      StepEnd end;
      attempt_dp45_fp64<kMetricKerr>(P, R, K, k1v, k7p, acc, h_used, end);
      if (acc) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          S[j][i] = xb[i];
          S[j][4 + i] = vb[i];
        }
        H[j] = h_used;
        if (Kst)
          for (int l = 0; l < 6; ++l)
#pragma unroll
            for (int i = 0; i < 4; ++i) Kst[j][l][i] = kl[l][i];
        if (end.xraw[2] < 0.0 || end.xraw[2] > kPi) *refl |= 1u << j;
        break;
      }
    }
  }
}

// The adjoint of one disk ray (sample idx) given dL/d(colour), its five
// sums added to acc5.
GG_DEV void backward_ray(const DevParams& P, const DiffOut& D, const double* dl_drgb,
                         uint64_t idx, double acc5[5]) {
  const DiffRay dr = D.rays[idx];
  if (dr.cls != kClsDisk || dr.n_acc == 0) return;
  const double dl[3] = {dl_drgb[3 * idx], dl_drgb[3 * idx + 1], dl_drgb[3 * idx + 2]};
  if (dl[0] == 0.0 && dl[1] == 0.0 && dl[2] == 0.0) return;
  const uint32_t n_ck = dr.n_ckpt < D.ckpt_per_ray ? dr.n_ckpt : D.ckpt_per_ray;
  const Ckpt* ck = D.ckpt + idx * D.ckpt_per_ray;
  double lam[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  double ga = 0.0, g_rin = 0.0, g_q = 0.0, g_sobs = 0.0;
  double S[kCkptEvery][8], H[kCkptEvery];
#if GG_ADJ_STORE_K
  double Kst[kCkptEvery][6][4];
#else
  double (*Kst)[6][4] = nullptr;
#endif
  bool ok = true;
  for (int seg = (int)n_ck - 1; seg >= 0 && ok; --seg) {
    const uint32_t first = (uint32_t)seg * kCkptEvery;
    const uint32_t steps = seg == (int)n_ck - 1 ? dr.n_acc - first : (uint32_t)kCkptEvery;
    if (steps == 0 || steps > (uint32_t)kCkptEvery) {
      ok = false;
      break;
    }
    uint32_t refl = 0;
    replay(P, ck[seg], steps, S, H, Kst, &refl);
    for (int j = (int)steps - 1; j >= 0; --j) {
      if (seg == (int)n_ck - 1 && j == (int)steps - 1) {
        ok = crossing_vjp(P, S[j], S[j] + 4, H[j], dl, lam, &ga, &g_rin, &g_q, &g_sobs);
        if (!ok) break;
        continue;
      }
      if (refl & (1u << j)) lam[2] = -lam[2];  // theta -> -theta or 2 pi - theta
      dp45_vjp(P, S[j], S[j] + 4, H[j], Kst ? Kst[j] : nullptr, lam, lam + 4, &ga);
    }
  }
  if (!ok) return;
  double u, v;
  sample_uv(P, idx, u, v);
  Dual<3> y0[8], sobs;
  camera_dual(P, u, v, y0, &sobs);
  double g3[3] = {ga, 0.0, 0.0};
#pragma unroll
  for (int p = 0; p < 3; ++p) {
    for (int j = 0; j < 8; ++j) g3[p] += lam[j] * y0[j].d[p];
    g3[p] += g_sobs * sobs.d[p];
  }
  acc5[0] += g3[0];
  acc5[1] += g3[1];
  acc5[2] += g3[2];
  acc5[3] += g_rin;
  acc5[4] += g_q;
}

// Work list of the backward pass: the disk rays with a nonzero dL/d(colour),
// longest first, by a counting sort on the checkpoint count (segments of
// kCkptEvery accepted steps).  Warps claim 32 rays of about equal length at a
// time (on the 512^2 image the lanes' useful share of a warp's steps goes from
// 0.78 to 1.0), and the longest chains, which set the pass's tail, start at
// once instead of in a later wave of blocks.
struct BackwardList {
  unsigned long long* head;  // next entry to claim
  uint32_t* total;           // entries in the list
  uint32_t* bins;            // per key: its count, then (after the scan) its next slot
  uint64_t* list;            // sample indices
  uint32_t n_keys;           // = D.ckpt_per_ray
};

constexpr int kScanThreads = 1024;

GG_DEV bool backward_key(const DiffOut& D, const double* dl, uint64_t idx, uint32_t* key) {
  const DiffRay dr = D.rays[idx];
  if (dr.cls != kClsDisk || dr.n_acc == 0) return false;
  if (dl[3 * idx] == 0.0 && dl[3 * idx + 1] == 0.0 && dl[3 * idx + 2] == 0.0) return false;
  uint32_t n_ck = dr.n_ckpt < D.ckpt_per_ray ? dr.n_ckpt : D.ckpt_per_ray;
  if (n_ck == 0) n_ck = 1;
  *key = D.ckpt_per_ray - n_ck;  // more segments, smaller key
  return true;
}

// Neighbouring disk rays mostly share a key: the lanes of a warp with the
// same key take their slots with one atomic (count and scatter), which keeps
// the popular bins from serialising.  The loops run the same trips on every
// lane of a block, so the warp-wide votes see all 32 lanes.
__global__ void backward_count_kernel(const __grid_constant__ DevParams P,
                                      const __grid_constant__ DiffOut D, const double* dl,
                                      BackwardList L) {
  const unsigned lane = threadIdx.x & 31u;
  for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < P.n_rays;
       base += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t idx = base + threadIdx.x;
    uint32_t k = 0;
    const bool has = idx < P.n_rays && backward_key(D, dl, idx, &k);
    const unsigned grp = __match_any_sync(kFull, has ? k : 0xffffffffu);
    if (has && lane == (unsigned)(__ffs(grp) - 1)) atomicAdd(L.bins + k, (uint32_t)__popc(grp));
  }
}

// Exclusive prefix sum of the key counts, in place, and the total (one block
// of kScanThreads threads, each over a contiguous run of keys).
__global__ void __launch_bounds__(kScanThreads) backward_scan_kernel(BackwardList L) {
  __shared__ uint32_t part[kScanThreads];
  const uint32_t t = threadIdx.x;
  const uint32_t per = (L.n_keys + kScanThreads - 1) / kScanThreads;
  const uint32_t b0 = t * per < L.n_keys ? t * per : L.n_keys;
  const uint32_t b1 = b0 + per < L.n_keys ? b0 + per : L.n_keys;
  uint32_t sum = 0;
  for (uint32_t b = b0; b < b1; ++b) sum += L.bins[b];
  part[t] = sum;
  __syncthreads();
  for (uint32_t off = 1; off < kScanThreads; off <<= 1) {
    const uint32_t v = t >= off ? part[t - off] : 0u;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  uint32_t run = t ? part[t - 1] : 0u;
  for (uint32_t b = b0; b < b1; ++b) {
    const uint32_t c = L.bins[b];
    L.bins[b] = run;
    run += c;
  }
  if (t == kScanThreads - 1) *L.total = part[t];
}

__global__ void backward_scatter_kernel(const __grid_constant__ DevParams P,
                                        const __grid_constant__ DiffOut D, const double* dl,
                                        BackwardList L) {
  const unsigned lane = threadIdx.x & 31u;
  for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < P.n_rays;
       base += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t idx = base + threadIdx.x;
    uint32_t k = 0;
    const bool has = idx < P.n_rays && backward_key(D, dl, idx, &k);
    const unsigned grp = __match_any_sync(kFull, has ? k : 0xffffffffu);
    if (has) {
      const unsigned leader = (unsigned)(__ffs(grp) - 1);
      uint32_t first = 0;
      if (lane == leader) first = atomicAdd(L.bins + k, (uint32_t)__popc(grp));
      first = __shfl_sync(grp, first, leader);
      L.list[first + (uint32_t)__popc(grp & lanemask_lt())] = idx;
    }
  }
}

// Persistent: each warp claims the next 32 entries of the sorted list.
__global__ void __launch_bounds__(128, GG_ADJ_MIN_BLOCKS) diff_backward_kernel(const __grid_constant__ DevParams P,
                                                            const __grid_constant__ DiffOut D,
                                                            const double* dl_drgb,
                                                            double* grad5, BackwardList L) {
  double acc5[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  const unsigned lane = threadIdx.x & 31u;
  const uint64_t n = *L.total;
  for (;;) {
    unsigned long long b = 0;
    if (lane == 0) b = atomicAdd(L.head, 32ull);
    b = __shfl_sync(kFull, b, 0);
    if (b >= n) break;
    if (b + lane < n) backward_ray(P, D, dl_drgb, L.list[b + lane], acc5);
  }
#pragma unroll
  for (int p = 0; p < 5; ++p) {
    double x = acc5[p];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31u) == 0 && x != 0.0) atomicAdd(grad5 + p, x);
  }
}

}  // namespace

size_t backward_list_bytes(uint64_t n_rays, uint32_t n_keys) {
  return 16 + ((4 * (size_t)n_keys + 7) & ~size_t(7)) + 8 * n_rays;
}

cudaError_t launch_diff_backward(const DevParams& P, const DiffOut& D, const double* dl_drgb,
                                 double* grad5, void* list_buf, int sms, cudaStream_t stream) {
  char* base = static_cast<char*>(list_buf);
  BackwardList L;
  L.head = reinterpret_cast<unsigned long long*>(base);
  L.total = reinterpret_cast<uint32_t*>(base + 8);
  L.bins = reinterpret_cast<uint32_t*>(base + 16);
  L.list = reinterpret_cast<uint64_t*>(base + 16 + ((4 * (size_t)D.ckpt_per_ray + 7) & ~size_t(7)));
  L.n_keys = D.ckpt_per_ray;
  cudaError_t e = cudaMemsetAsync(base, 0, 16 + 4 * (size_t)D.ckpt_per_ray, stream);
  if (e != cudaSuccess) return e;
  const uint64_t blocks_needed = (P.n_rays + 255) / 256;
  uint64_t grid = (uint64_t)sms * 8;
  if (grid > blocks_needed) grid = blocks_needed;
  if (grid < 1) grid = 1;
  backward_count_kernel<<<(unsigned)grid, 256, 0, stream>>>(P, D, dl_drgb, L);
  backward_scan_kernel<<<1, kScanThreads, 0, stream>>>(L);
  backward_scatter_kernel<<<(unsigned)grid, 256, 0, stream>>>(P, D, dl_drgb, L);
  int bps = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, diff_backward_kernel, 128, 0);
  if (e != cudaSuccess) return e;
  diff_backward_kernel<<<sms * (bps > 0 ? bps : 1), 128, 0, stream>>>(P, D, dl_drgb, grad5, L);
  return cudaGetLastError();
}

}  // namespace gg
