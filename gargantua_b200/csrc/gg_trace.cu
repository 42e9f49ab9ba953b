// gg_trace.cu -- persistent ray-tracing kernels for sm_100a.
//
// Work decomposition.  A render is a flat queue of n = width*height*spp
// samples.  The grid is persistent (a few CTAs per SM, sized from the
// occupancy of the instantiation); each warp takes 32 sample indices from a
// global counter at a time and hands them to its lanes as they free up.
// After every `kPeriod` RK45 attempts the warp ballots which lanes finished
// and refills exactly those lanes, so a warp keeps all 32 lanes busy even
// though per-ray attempt counts differ by 100x between a ray that escapes
// directly and one that grazes the photon sphere.  Ray state stays in
// registers from the camera to the terminal surface; HBM only sees the
// finished outcome (and, for supersampling, one linear colour per sample).
#include <cuda_runtime.h>

#include <cstdint>

#include "gg_device.cuh"
#include "gg_launch.h"
#include "gg_scene.cuh"
#include "gg_trace_common.cuh"

namespace gg {

namespace {

// A ray in the FP64 pass of the mixed form goes back to the FP32 stepper
// once an accepted step leaves it this far outside the band: r beyond
// band_r + kBackMargin M and theta more than kBackPole * pole_band from
// both poles (the margin keeps rays from bouncing between the passes).
// Measured on the 1080p Kerr frame (median ms; the endpoint error and class
// agreement identical throughout): margin / pole factor 0.5 / 1.5: 27.8,
// 1 / 2: 27.6, 1 / 3: 27.7, 2 / 2: 27.1, 2 / 3: 27.2, 3 / 4: 27.4,
// 5 / 6: 27.3, 8 / 8: 27.9.  With 2 M no ray re-enters the band.
#ifndef GG_BACK_MARGIN
#define GG_BACK_MARGIN 2.0
#endif
#ifndef GG_BACK_POLE
#define GG_BACK_POLE 2.0
#endif
constexpr double kBackMargin = GG_BACK_MARGIN;
constexpr double kBackPole = GG_BACK_POLE;

// Writes a ray clear of the band to the return queue (out of line, once per
// returned ray).
__device__ __noinline__ void hand_back(const DevOutputs& O, DevControl* ctl, Ray R, uint64_t idx,
                                       uint32_t n_att, uint32_t n_acc, uint32_t scene) {
  const unsigned long long slot = atomicAdd(&ctl->returned, 1ull);
  if (slot >= O.ret_cap) {
    atomicExch(&ctl->queue_overflow, 1u);
    return;
  }
  QueuedRay& q = O.ret[slot];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    q.x[i] = R.x[i];
    q.v[i] = R.v[i];
  }
  q.h = R.h;
  q.lam = R.lam;
  q.idx = idx;
  q.n_att = n_att;
  q.n_acc = n_acc;
  q.scene = scene;
}

// SRC: kSrcCamera traces the render's samples from the camera; kSrcQueue
// finishes, in FP64, the rays the mixed-precision pass handed over (their
// count is read from ctl->queued, which that pass wrote before this launch);
// with P.hand_back it returns rays that leave the band to the mixed form.
// BATCH (kSrcQueue only): the rays come from a batched render; each carries
// its scene, whose parameters and outputs are in B.  SCENE (kSrcCamera, no
// thin disk): every accepted step's chord is tested against P's scene of
// objects first.  CKPT (kSrcCamera, Kerr, thin disk, full Dormand-Prince):
// the differentiable render's forward, which also stores each ray's state
// (x, v, next h) at its start and after every kCkptEvery-th accepted step it
// survives (O.ckpt) and, when it ends, its DiffRay (O.diff_rays).
template <int METRIC, int DISK, int STEPPER, int SRC, bool BATCH, bool SCENE, bool CKPT,
          bool SMALL>
__global__ void __launch_bounds__(kTraceBlock,
                                  METRIC != kMetricKerr                 ? kTraceMinBlocksSchw
                                  : (SRC == kSrcQueue || CKPT || SMALL) ? kTraceMinBlocksKerrChain
                                                                        : kTraceMinBlocksKerr)
    trace_fp64_kernel(const __grid_constant__ DevParams P, const __grid_constant__ DevOutputs O,
                      DevControl* ctl, const __grid_constant__ BatchTable B) {
  const unsigned lane = threadIdx.x & 31u;
  const uint64_t n_src =
      SRC == kSrcQueue ? (ctl->queued < O.queue_cap ? ctl->queued : O.queue_cap) : P.n_rays;
  unsigned long long* const head = SRC == kSrcQueue ? &ctl->next_queued : &ctl->next_ray;
  __shared__ BlockStats bs;
  __shared__ double k_smem[7][4][kTraceBlock];  // stage derivatives, see KStore
  const KStore K{k_smem};
  if (threadIdx.x < sizeof(BlockStats) / 8)
    reinterpret_cast<unsigned long long*>(&bs)[threadIdx.x] = 0ull;
  __syncthreads();
  auto finish = [&](const DevParams& pp, const DevOutputs& oo, uint64_t i, int cls, const Ray& r,
                    uint32_t na, uint32_t nc, double inten_o, double temp_o, bool cr,
                    double sky_th, double sky_ph) {
    finish_sample(pp, oo, i, cls, r, na, nc, inten_o, temp_o, cr, sky_th, sky_ph);
    atomicAdd(&bs.attempts, (unsigned long long)na);
    atomicAdd(&bs.accepted, (unsigned long long)nc);
    atomicAdd(&bs.cls[cls], 1ull);
  };
  uint32_t n_att0 = 0;  // kSrcQueue: attempts the ray had made before the hand-off

  Ray R;
  uint64_t idx = 0;
  uint32_t scene = 0;  // BATCH: the ray's scene
  bool live = false;
  uint32_t n_att = 0, n_acc = 0;
  double inten = 0.0, trans = 1.0;  // volumetric disk accumulators
  bool crossed = false;
  bool k1_valid = false;    // K(0, .) holds a(x, v) of the current state
  bool k7_pending = false;  // full DP: K(6, .) is the next k1, copy pending
  uint32_t n_ckpt = 0;      // CKPT: checkpoints of the ray so far
  auto save_ckpt = [&]() {
    if (n_ckpt < O.ckpt_per_ray) {
      Ckpt& c = O.ckpt[idx * O.ckpt_per_ray + n_ckpt];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        c.x[i] = R.x[i];
        c.v[i] = R.v[i];
      }
      c.h = R.h;
    }
    ++n_ckpt;
  };

  uint64_t wbase = 0;
  uint32_t wcount = 0;
  bool wdone = false;
  unsigned budget_pending = 0;

  for (;;) {
    // ---- refill lanes whose ray finished ----------------------------------
    unsigned need = __ballot_sync(kFull, !live);
    if (P.attempt_budget && need && !wdone) {
      unsigned long long ab = 0;
      if (lane == 0) ab = atomicOr(&ctl->abort, 0u);
      if (__shfl_sync(kFull, ab, 0)) wdone = true;
    }
    while (need && !wdone) {
      if (wcount == 0) {
        unsigned long long b = 0;
        if (lane == 0) {
          b = atomicAdd(head, (unsigned long long)kChunk);
          if (P.attempt_budget) {
            const unsigned long long used = atomicAdd(&ctl->budget_used, 0ull);
            if (used > P.attempt_budget) {
              atomicExch(&ctl->abort, 1u);
              b = n_src;  // stop taking work
            }
          }
        }
        b = __shfl_sync(kFull, b, 0);
        if (b >= n_src) {
          wdone = true;
          break;
        }
        wbase = b;
        const uint64_t left = n_src - b;
        wcount = left < kChunk ? (uint32_t)left : kChunk;
      }
      const unsigned nn = (unsigned)__popc(need);
      const unsigned take = nn < wcount ? nn : wcount;
      const unsigned rank = (unsigned)__popc(need & lanemask_lt());
      if (!live && rank < take) {
        if (SRC == kSrcQueue) {
          const QueuedRay& q = O.queue[wbase + rank];
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            R.x[i] = q.x[i];
            R.v[i] = q.v[i];
          }
          R.h = q.h;
          R.lam = q.lam;
          idx = q.idx;
          if (BATCH) scene = q.scene;
          n_att = n_att0 = q.n_att;
          n_acc = q.n_acc;
        } else {
          idx = camera_sample(P, wbase + rank);
          R = start_sample(P, idx);
          n_att = 0;
          n_acc = 0;
          if (CKPT) {
            n_ckpt = 0;
            save_ckpt();
          }
        }
        live = true;
        inten = 0.0;
        trans = 1.0;
        crossed = false;
        k1_valid = false;
        k7_pending = false;
      }
      wbase += take;
      wcount -= take;
      need = __ballot_sync(kFull, !live);
    }
    if (!__any_sync(kFull, live)) break;

    // ---- advance every live ray by up to kPeriod attempts -----------------
#pragma unroll 1
    for (int it = 0; it < (SRC == kSrcQueue ? kQueuePeriod : kPeriod); ++it) {
      if (!live) continue;
      // this lane's scene: the batch's entry, or the render's own parameters
      const DevParams& PL = BATCH ? B.scenes[scene].P : P;
      const DevOutputs& OL = BATCH ? B.scenes[scene].O : O;
      double xb[4], vb[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        xb[i] = R.x[i];
        vb[i] = R.v[i];
      }
      const double lam_b = R.lam;
      bool acc;
      double h_used = 0.0;
      StepEnd end;
      int res;
      if (STEPPER == kStepperDP45)
        res = attempt_dp45_fp64<METRIC>(PL, R, K, k1_valid, k7_pending, acc, h_used, end);
      else
        res = attempt_fp64<METRIC>(PL, R, K, k1_valid, acc, h_used);
      n_att += 1;
      if (acc) n_acc += 1;
      int done_cls = -1;
      double out_int = 0.0, out_temp = 0.0;
      // full Dormand-Prince, checkerboard sky, thin disk or none: the sky is
      // read where the ray meets the escape sphere (sky_at_cross)
      constexpr bool kSkyCross = STEPPER == kStepperDP45 && DISK != kDiskVolumetric;
      bool sky_at_cross = false;
      double sky_th = 0.0, sky_ph = 0.0;
      double scene_rgb[3];

      if (SCENE && acc) {
        // trace_ray_with_scene (tracer.rs:218-236): the chord between the
        // step's ends, in Cartesian coordinates, against the scene
        double cb[3], ca[3], dd[3];
        sph_to_cart(xb, cb);
        sph_to_cart(R.x, ca);
#pragma unroll
        for (int i = 0; i < 3; ++i) dd[i] = sub_rn(ca[i], cb[i]);
        if (dot3_nc(dd, dd) > 0.0) {
          double t_hit;
          const int k = scene_nearest(PL, cb, dd, t_hit);
          if (k >= 0) {
            scene_shade<METRIC>(PL, k, t_hit, cb, dd, scene_rgb);
            if (DISK == kDiskVolumetric) {  // tracer.rs:293-309
              double dl[3];
              disk_color(inten, dl);
#pragma unroll
              for (int c = 0; c < 3; ++c) scene_rgb[c] = add_rn(mul_rn(scene_rgb[c], trans), dl[c]);
            }
            done_cls = kClsScene;
          }
        }
      }

      if (acc && done_cls < 0) {
        // The step's path: the reference's Euler segment (exactly linear in
        // the step fraction), or the full Dormand-Prince step's continuous
        // extension.
        double raw[4];
#pragma unroll
        for (int i = 0; i < 4; ++i)
          raw[i] = STEPPER == kStepperDP45 ? end.xraw[i] : xb[i] + h_used * vb[i];
        const bool esc = (OL.cross || (kSkyCross && PL.sky == kSkyChecker)) &&
                         xb[1] <= PL.max_radius && raw[1] > PL.max_radius;
        double d_b = 0.0, d_a = 0.0;
        bool dsk = false;
        if (DISK == kDiskThin) {
          d_b = xb[2] - kHalfPi;
          d_a = R.x[2] - kHalfPi;
          dsk = (d_b < 0.0 && d_a >= 0.0) || (d_b > 0.0 && d_a <= 0.0);
        }
        if (esc || dsk) {
          StepSpan sp;
          if (STEPPER == kStepperDP45) {
#pragma unroll
            for (int i = 0; i < 4; ++i) {
              sp.xb[i] = xb[i];
              sp.vb[i] = vb[i];
              sp.xa[i] = raw[i];
              sp.va[i] = R.v[i];
            }
            for (int l = 0; l < 7; ++l)
#pragma unroll
              for (int i = 0; i < 4; ++i) sp.k[l][i] = K(l, i);
            sp.h = h_used;
          }
          // state c where component `comp` meets `target`; returns the step
          // fraction (the reference stepper's is linear_s, on its segment)
          auto cross_at = [&](int comp, double target, double linear_s, double c[8]) {
            if (STEPPER == kStepperDP45) {
              const double s = dense_crossing(sp, comp, target, c);
              normalize_coords(c);
              return s;
            }
            segment_point(xb, vb, h_used, R.v, linear_s, c);
            return linear_s;
          };
          if (esc) {
            double c[8];
            cross_at(1, PL.max_radius, (PL.max_radius - xb[1]) / (raw[1] - xb[1]), c);
            if (OL.cross) {
              store_cross(PL, OL, idx, c);
              crossed = true;
            }
            if (kSkyCross && PL.sky == kSkyChecker) {
              sky_at_cross = true;
              sky_th = c[2];
              sky_ph = c[3];
            }
          }
          if (dsk) {
            double c[8];
            const double s = cross_at(2, kHalfPi, d_b / (d_b - d_a), c);
            const double r_c =
                STEPPER == kStepperDP45 ? c[1] : xb[1] + s * (raw[1] - xb[1]);
            if (r_c >= PL.r_inner && r_c <= PL.r_outer) {
              c[1] = r_c;
              c[2] = kHalfPi;
              const double g = redshift_factor<METRIC>(PL, r_c, kHalfPi, c + 4);
              const double q = PL.r_inner / r_c;
              const double g2 = g * g;
              out_int = (g2 * g2) * pow(q, PL.emissivity_index);
              out_temp = g * pow(q, 0.75);
#pragma unroll
              for (int i = 0; i < 4; ++i) {
                R.x[i] = c[i];
                R.v[i] = c[4 + i];
              }
              R.lam = lam_b + s * h_used;
              store_cross(PL, OL, idx, c);
              crossed = true;
              done_cls = kClsDisk;
            }
          }
        }
        // Beyond the escape sphere the next attempt only finds r > max_radius
        // and returns Escaped; the ray ends here, counting that attempt.
        if (sky_at_cross && done_cls < 0 && n_att < PL.max_steps) {
          n_att += 1;
          done_cls = kClsEscaped;
        }
      }
      if (DISK == kDiskVolumetric && done_cls < 0) {
        // trace_ray_with_disk (tracer.rs:96-145)
        const double dlambda = fmax(R.lam - lam_b, 0.0);
        if (dlambda > 0.0) {
          double mid[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) mid[i] = 0.5 * (xb[i] + R.x[i]);
          double sn, cs;
          sincos(mid[2], &sn, &cs);
          const double cap_r = mid[1] * fabs(sn);
          const double z = mid[1] * cs;
          if (!(cap_r < PL.r_inner || cap_r > PL.r_outer)) {
            const double qq = PL.r_inner / cap_r;
            const double rho = PL.density_0 * (qq * qq) *
                               exp(-z * z / (2.0 * PL.scale_height * PL.scale_height));
            if (rho > 0.0) {
              const double j = rho * rho * pow(qq, 0.75);
              double pm[4];
#pragma unroll
              for (int i = 0; i < 4; ++i) pm[i] = 0.5 * (vb[i] + R.v[i]);
              const double g = redshift_factor<METRIC>(PL, mid[1], mid[2], pm);
              const double g2 = g * g;
              inten = inten + j * (g2 * g2) * dlambda * trans;
              trans = trans * exp(-rho * dlambda * 0.1);
              if (trans < 1e-3) {
                done_cls = kClsDisk;
                out_int = inten;
                out_temp = PL.temperature_0;
              }
            }
          }
        }
        if (done_cls < 0 && res != kContinue) {
          if (inten > 0.0) {
            done_cls = kClsDisk;
            out_int = inten;
            out_temp = PL.temperature_0;
          } else {
            done_cls = res == kEscaped ? kClsEscaped : kClsHorizon;
          }
        }
        if (done_cls < 0 && n_att >= PL.max_steps) {
          if (inten > 0.0) {
            done_cls = kClsDisk;
            out_int = inten;
            out_temp = PL.temperature_0;
          } else {
            done_cls = kClsMaxSteps;
          }
        }
      } else if (done_cls < 0) {
        if (res == kHorizon) done_cls = kClsHorizon;
        else if (res == kEscaped) done_cls = kClsEscaped;
        else if (n_att >= PL.max_steps) done_cls = kClsMaxSteps;
      }
      // a checkpoint after every kCkptEvery-th accepted step that did not end
      // the ray at a crossing (a step that runs out of attempts still counts)
      if (CKPT && acc && (done_cls < 0 || done_cls == kClsMaxSteps) &&
          n_acc % kCkptEvery == 0)
        save_ckpt();
      if (SRC == kSrcQueue && P.hand_back && acc && done_cls < 0 &&
          R.x[1] > (double)PL.band_r + kBackMargin &&
          fmin(R.x[2], kPi - R.x[2]) > kBackPole * (double)PL.pole_band) {
        hand_back(O, ctl, R, idx, n_att, n_acc, scene);
        atomicAdd(&bs.fp64_att, (unsigned long long)(n_att - n_att0));
        live = false;
        continue;
      }
      if (SCENE && done_cls == kClsScene) {
        finish_scene_sample(PL, OL, idx, R, n_att, n_acc, inten, scene_rgb);
        atomicAdd(&bs.attempts, (unsigned long long)n_att);
        atomicAdd(&bs.accepted, (unsigned long long)n_acc);
        atomicAdd(&bs.cls[kClsScene], 1ull);
        budget_pending += n_att;
        live = false;
      } else if (done_cls >= 0) {
        finish(PL, OL, idx, done_cls, R, n_att, n_acc, out_int, out_temp, crossed,
               sky_at_cross ? sky_th : R.x[2], sky_at_cross ? sky_ph : R.x[3]);
        if (CKPT) O.diff_rays[idx] = DiffRay{n_acc, n_ckpt, done_cls, 0u};
        if (SRC == kSrcQueue) atomicAdd(&bs.fp64_att, (unsigned long long)(n_att - n_att0));
        budget_pending += n_att;
        live = false;
      }
    }
    if (P.attempt_budget) {
      // account finished work; stop live rays once the budget is gone
      const unsigned long long wsum = __reduce_add_sync(kFull, budget_pending);
      budget_pending = 0;
      unsigned ab = 0;
      if (lane == 0) {
        const unsigned long long used = atomicAdd(&ctl->budget_used, wsum) + wsum;
        if (used > P.attempt_budget) atomicExch(&ctl->abort, 1u);
        ab = atomicOr(&ctl->abort, 0u);
      }
      if (__shfl_sync(kFull, ab, 0)) {
        wdone = true;
        if (live) {
          finish(BATCH ? B.scenes[scene].P : P, BATCH ? B.scenes[scene].O : O, idx, kClsBudget,
                 R, n_att, n_acc, 0.0, 0.0, crossed, R.x[2], R.x[3]);
          if (SRC == kSrcQueue) atomicAdd(&bs.fp64_att, (unsigned long long)(n_att - n_att0));
          live = false;
        }
      }
    }
  }

  // ---- per-block statistics -----------------------------------------------
  __syncthreads();
  if (threadIdx.x == 0) {
    atomicAdd(&ctl->attempts, bs.attempts);
    atomicAdd(&ctl->accepted, bs.accepted);
    if (SRC == kSrcQueue && bs.fp64_att) atomicAdd(&ctl->fp64_attempts, bs.fp64_att);
#pragma unroll
    for (int k = 0; k < kNumClasses; ++k)
      if (bs.cls[k]) atomicAdd(&ctl->class_count[k], bs.cls[k]);
  }
}

// Averages the spp linear sample colours of each pixel in sample order and
// encodes sRGB (render_row, renderer.rs:326-343).
__global__ void reduce_samples_kernel(const __grid_constant__ DevParams P, const double* samples,
                                      uint8_t* rgb8) {
  const uint64_t n_pix = (uint64_t)P.width * P.rows;
  for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n_pix;
       p += (uint64_t)gridDim.x * blockDim.x) {
    double acc[3] = {0.0, 0.0, 0.0};
    const double* s = samples + 3 * p * P.spp;
    for (uint32_t k = 0; k < P.spp; ++k) {
#pragma unroll
      for (int c = 0; c < 3; ++c) acc[c] = add_rn(acc[c], s[3 * k + c]);
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) rgb8[3 * p + c] = encode_channel(mul_rn(acc[c], P.inv_spp));
  }
}

template <int METRIC, int DISK, int STEPPER, int SRC, bool BATCH = false, bool SCENE = false,
          bool CKPT = false, bool SMALL = false>
const void* trace_fn() {
  return reinterpret_cast<const void*>(
      &trace_fp64_kernel<METRIC, DISK, STEPPER, SRC, BATCH, SCENE, CKPT, SMALL>);
}

// Kerr camera passes of fewer samples than this run the 4-CTA budget of the
// chain-bound passes: a few rays per lane, so the longest rays set the time.
constexpr uint64_t kSmallRender = 1ull << 20;

// With a scene: no disk or the volumetric one (the reference's
// render_with_scene and render_with_disk_and_scene).
template <int STEPPER, bool SMALL>
const void* select_scene_kerr(const DevParams& P) {
  return P.disk == kDiskVolumetric
             ? trace_fn<kMetricKerr, kDiskVolumetric, STEPPER, kSrcCamera, false, true, false,
                        SMALL>()
             : trace_fn<kMetricKerr, kDiskNone, STEPPER, kSrcCamera, false, true, false, SMALL>();
}

template <int STEPPER>
const void* select_scene(const DevParams& P) {
  if (P.metric == kMetricKerr)
    return P.n_rays < kSmallRender ? select_scene_kerr<STEPPER, true>(P)
                                   : select_scene_kerr<STEPPER, false>(P);
  return P.disk == kDiskVolumetric
             ? trace_fn<kMetricSchwarzschild, kDiskVolumetric, STEPPER, kSrcCamera, false, true>()
             : trace_fn<kMetricSchwarzschild, kDiskNone, STEPPER, kSrcCamera, false, true>();
}

template <int STEPPER, bool SMALL>
const void* select_disk_kerr(const DevParams& P) {
  if (P.disk == kDiskThin)
    return trace_fn<kMetricKerr, kDiskThin, STEPPER, kSrcCamera, false, false, false, SMALL>();
  if (P.disk == kDiskVolumetric)
    return trace_fn<kMetricKerr, kDiskVolumetric, STEPPER, kSrcCamera, false, false, false,
                    SMALL>();
  return trace_fn<kMetricKerr, kDiskNone, STEPPER, kSrcCamera, false, false, false, SMALL>();
}

template <int STEPPER>
const void* select_metric_disk(const DevParams& P) {
  if (P.scene) return select_scene<STEPPER>(P);
  if (P.metric == kMetricKerr)
    return P.n_rays < kSmallRender ? select_disk_kerr<STEPPER, true>(P)
                                   : select_disk_kerr<STEPPER, false>(P);
  if (P.disk == kDiskThin) return trace_fn<kMetricSchwarzschild, kDiskThin, STEPPER, kSrcCamera>();
  if (P.disk == kDiskVolumetric)
    return trace_fn<kMetricSchwarzschild, kDiskVolumetric, STEPPER, kSrcCamera>();
  return trace_fn<kMetricSchwarzschild, kDiskNone, STEPPER, kSrcCamera>();
}

const void* select_trace(const DevParams& P) {
  // gg_forward_ckpt admits only Kerr, the thin disk and the full stepper
  if (P.ckpt)
    return trace_fn<kMetricKerr, kDiskThin, kStepperDP45, kSrcCamera, false, false, true>();
  return P.stepper == kStepperDP45 ? select_metric_disk<kStepperDP45>(P)
                                   : select_metric_disk<kStepperReference>(P);
}

// The FP64 pass of the mixed form: full Dormand-Prince, thin disk or none.
template <bool BATCH>
const void* select_queue_trace_b(const DevParams& P) {
  if (P.metric == kMetricKerr)
    return P.disk == kDiskThin
               ? trace_fn<kMetricKerr, kDiskThin, kStepperDP45, kSrcQueue, BATCH>()
               : trace_fn<kMetricKerr, kDiskNone, kStepperDP45, kSrcQueue, BATCH>();
  return P.disk == kDiskThin
             ? trace_fn<kMetricSchwarzschild, kDiskThin, kStepperDP45, kSrcQueue, BATCH>()
             : trace_fn<kMetricSchwarzschild, kDiskNone, kStepperDP45, kSrcQueue, BATCH>();
}

const void* select_queue_trace(const DevParams& P, bool batch) {
  return batch ? select_queue_trace_b<true>(P) : select_queue_trace_b<false>(P);
}

}  // namespace

cudaError_t trace_occupancy(const DevParams& P, int* blocks_per_sm) {
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, select_trace(P),
                                                       kTraceBlock, 0);
}

cudaError_t queue_trace_occupancy(const DevParams& P, int* blocks_per_sm) {
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      blocks_per_sm, select_queue_trace(P, false), kTraceBlock, 0);
}

cudaError_t launch_queue_trace(const DevParams& P, const DevOutputs& O, DevControl* ctl,
                               int grid, cudaStream_t stream, const BatchTable* batch) {
  const void* fn = select_queue_trace(P, batch != nullptr);
  DevParams p = P;
  DevOutputs o = O;
  BatchTable b{};
  if (batch) b = *batch;
  void* args[] = {&p, &o, &ctl, &b};
  return cudaLaunchKernel(fn, dim3(grid), dim3(kTraceBlock), args, 0, stream);
}

cudaError_t launch_trace(const DevParams& P, const DevOutputs& O, DevControl* ctl, int grid,
                         cudaStream_t stream) {
  const void* fn = select_trace(P);
  DevParams p = P;
  DevOutputs o = O;
  BatchTable b{};
  void* args[] = {&p, &o, &ctl, &b};
  return cudaLaunchKernel(fn, dim3(grid), dim3(kTraceBlock), args, 0, stream);
}

// Between the rounds of the mixed form: the band queue's entries are all
// consumed; its count moves to the running total and it restarts empty.
__global__ void next_round_kernel(DevControl* ctl) {
  ctl->band_total += ctl->queued;
  ctl->queued = 0;
  ctl->next_queued = 0;
}

cudaError_t launch_next_round(DevControl* ctl, cudaStream_t stream) {
  next_round_kernel<<<1, 1, 0, stream>>>(ctl);
  return cudaGetLastError();
}

cudaError_t launch_reduce(const DevParams& P, const double* samples, uint8_t* rgb8, int sms,
                          cudaStream_t stream) {
  const uint64_t n_pix = (uint64_t)P.width * P.rows;
  uint64_t blocks = (n_pix + 255) / 256;
  const uint64_t cap = (uint64_t)sms * 8;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  reduce_samples_kernel<<<(unsigned)blocks, 256, 0, stream>>>(P, samples, rgb8);
  return cudaGetLastError();
}

}  // namespace gg
