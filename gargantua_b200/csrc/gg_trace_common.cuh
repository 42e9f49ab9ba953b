// gg_trace_common.cuh -- lane bookkeeping shared by the persistent trace
// kernels (the FP64 kernel in gg_trace.cu, the mixed-precision kernel in
// gg_mixed.cu): work-queue constants, sample setup and finishing, per-block
// statistics and the crossing-state output.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "gg_device.cuh"
#include "gg_launch.h"

namespace gg {

namespace {

constexpr unsigned kFull = 0xffffffffu;
// Attempts between refills: the FP64 kernel's and the mixed kernel's
// (single-scene renders; batches autotune theirs).  Measured on the 1080p
// Kerr frame, FP64 drop-in / mixed ms: period 2: 52.9 / 33.4, 4: 49.9 / 31.1,
// 8: 47.0 / 29.3, 16: 45.3 / 29.2, 32: 44.3 / 29.4 (fewer ballots and
// refills; lanes that finish early wait longer).  Measured again for the mixed
// camera pass at 8 / 16 / 32 (the current build): 1080p 25.6 / 25.7 / 25.9
// ms, the stress view at 2048^2 x 4 spp 83.9 / 82.2 / 84.9 ms, the full stress
// frame 1.273 / 1.249 / 1.306 s.
#ifndef GG_TRACE_PERIOD
#define GG_TRACE_PERIOD 32
#endif
#ifndef GG_MIXED_PERIOD
#define GG_MIXED_PERIOD 16
#endif
// The mixed form's FP64 band passes refill more often: on views whose band
// holds many rays of uneven length the pass is throughput-bound, and idle
// lanes cost more than ballots.  Measured (period 32 / 16 / 8 / 4 / 2): the
// stress view at 2048^2 x 4 spp 84.1 / 82.4 / 81.9 / 82.2 / 82.8 ms, the full
// stress frame 1.282 / 1.254 / 1.248 / 1.250 / 1.258 s, the 2,048-scene batch
// 2.376 / 2.357 / 2.350 / 2.357 / 2.357 s; the 1080p frame, whose band pass
// is one wave, 25.7 ms throughout.
#ifndef GG_QUEUE_PERIOD
#define GG_QUEUE_PERIOD 8
#endif
constexpr int kPeriod = GG_TRACE_PERIOD;
constexpr int kQueuePeriod = GG_QUEUE_PERIOD;
constexpr int kMixedPeriod = GG_MIXED_PERIOD;
constexpr uint32_t kChunk = 32;  // samples a warp takes from the queue at once

GG_DEV unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Work order of a camera pass: with GG_CENTER_OUT the traced rows are handed
// out from the middle outwards (m, m-1, m+1, m-2, ... with m = rows / 2),
// each row's samples in order; otherwise row by row from the top.  A view of
// the hole has its costliest rays (the shadow's edge, the photon ring) in the
// middle; started first, they no longer end a pass alone.  Outputs stay at
// each sample's own index.  Measured, row order / middle out (ms): the
// reference CLI's 800 x 600 render with the lensed spheres 17.9 / 15.8, with
// the volumetric disk 15.9 / 14.6, Kerr with a sky map 26.6 / 24.9; the mixed
// 1080p Kerr frame 27.7 / 27.4; FP64 1080p and the adjoint unchanged.
#ifndef GG_CENTER_OUT
#define GG_CENTER_OUT 1
#endif
GG_DEV uint64_t camera_sample(const DevParams& P, uint64_t w) {
  if (!GG_CENTER_OUT) return w;
  const uint64_t per_row = (uint64_t)P.width * P.spp;
  const uint64_t k = w / per_row;
  const uint64_t m = P.rows / 2;
  const uint64_t row = (k & 1) ? m - (k + 1) / 2 : m + k / 2;
  return row * per_row + (w - k * per_row);
}

// Writes the finished sample's outcome and colour.  Runs once per ray, so it
// is kept out of line: its shading code (several pow) would otherwise sit in
// the hot stepping loop's instruction footprint.  (sky_th, sky_ph) is where
// the checkerboard sky is read: the final position, or, for the full
// Dormand-Prince stepper, the escape-sphere crossing.
GG_DEV void write_outcome(const DevParams& P, const DevOutputs& O, uint64_t idx, int cls,
                          const Ray& R, uint32_t n_att, uint32_t n_acc, double intensity,
                          double color_temp, bool crossed, const double lin[3]) {
  {
    const uint64_t n = P.n_rays;
    if (O.cls) O.cls[idx] = cls;
    if (O.x) {
#pragma unroll
      for (int c = 0; c < 4; ++c) O.x[c * n + idx] = R.x[c];
    }
    if (O.v) {
#pragma unroll
      for (int c = 0; c < 4; ++c) O.v[c * n + idx] = R.v[c];
    }
    if (O.lam) O.lam[idx] = R.lam;
    if (O.attempts) O.attempts[idx] = n_att;
    if (O.accepted) O.accepted[idx] = n_acc;
    if (O.intensity) O.intensity[idx] = intensity;
    if (O.color_temp) O.color_temp[idx] = color_temp;
    if (O.rgb) {
#pragma unroll
      for (int c = 0; c < 3; ++c) O.rgb[3 * idx + c] = lin[c];
    }
    if (O.cross && !crossed) {
      const double qnan = __longlong_as_double(0x7ff8000000000000LL);
#pragma unroll
      for (int c = 0; c < 8; ++c) O.cross[c * n + idx] = qnan;
    }
    if (O.sample_rgb) {
#pragma unroll
      for (int c = 0; c < 3; ++c) O.sample_rgb[3 * idx + c] = lin[c];
    } else if (O.rgb8) {
#pragma unroll
      for (int c = 0; c < 3; ++c) O.rgb8[3 * idx + c] = encode_channel(lin[c]);
    }
  }
}

__device__ __noinline__ void finish_sample(const DevParams& P, const DevOutputs& O, uint64_t idx,
                                           int cls, Ray R, uint32_t n_att, uint32_t n_acc,
                                           double intensity, double color_temp, bool crossed,
                                           double sky_th, double sky_ph) {
  double lin[3];
  if (cls == kClsHorizon || cls == kClsBudget) {
    lin[0] = lin[1] = lin[2] = 0.0;
  } else if (cls == kClsEscaped) {
    if (P.sky == kSkyChecker)
      checker_sky(P, sky_th, sky_ph, lin);
    else if (P.sky == kSkyHdri)
      hdri_sky(P, R.v, lin);
    else
      procedural_sky(R.v, lin);
  } else if (cls == kClsDisk) {
    disk_color(intensity, lin);
  } else {
    lin[0] = 0.0;
    lin[1] = 0.0;
    lin[2] = 10.0 / 255.0;
  }
  write_outcome(P, O, idx, cls, R, n_att, n_acc, intensity, color_temp, crossed, lin);
}

// A ray whose chord hit the scene (RayOutcome::Scene): its colour was
// shaded at the hit; `intensity` is the volumetric disk's up to the hit.
__device__ __noinline__ void finish_scene_sample(const DevParams& P, const DevOutputs& O,
                                                 uint64_t idx, Ray R, uint32_t n_att,
                                                 uint32_t n_acc, double intensity,
                                                 const double rgb[3]) {
  const double lin[3] = {rgb[0], rgb[1], rgb[2]};
  write_outcome(P, O, idx, kClsScene, R, n_att, n_acc, intensity, 0.0, false, lin);
}

// Camera ray of sample idx (once per ray, out of line like finish_sample).
__device__ __noinline__ Ray start_sample(const DevParams& P, uint64_t idx) {
  double u, v;
  sample_uv(P, idx, u, v);
  Ray R;
  init_ray(P, u, v, R);
  return R;
}

// Per-block totals of the statistics (one shared-memory atomic per finished
// ray instead of per-thread counters, which would cost registers in the
// stepping loop); flushed to DevControl when the block exits.
struct BlockStats {
  unsigned long long attempts, accepted, cls[kNumClasses], fp64_att;
};

enum : int { kSrcCamera = 0, kSrcQueue = 1 };

// Point at fraction s of the last accepted Euler segment (the reference moves
// x by h*v_before, geodesic.rs:312, so x is linear in s); v interpolated.
GG_DEV void segment_point(const double xb[4], const double vb[4], double h, const double va[4],
                          double s, double out[8]) {
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const double raw = xb[i] + h * vb[i];
    out[i] = xb[i] + s * (raw - xb[i]);
    out[4 + i] = vb[i] + s * (va[i] - vb[i]);
  }
  normalize_coords(out);
}

GG_DEV void store_cross(const DevParams& P, const DevOutputs& O, uint64_t idx,
                        const double c[8]) {
  if (!O.cross) return;
#pragma unroll
  for (int i = 0; i < 8; ++i) O.cross[i * P.n_rays + idx] = c[i];
}

}  // namespace

}  // namespace gg
