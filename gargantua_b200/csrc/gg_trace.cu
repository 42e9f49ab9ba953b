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

namespace gg {

namespace {

constexpr unsigned kFull = 0xffffffffu;
#ifndef GG_TRACE_PERIOD
#define GG_TRACE_PERIOD 4
#endif
constexpr int kPeriod = GG_TRACE_PERIOD;  // attempts between refills
constexpr uint32_t kChunk = 32;  // samples a warp takes from the queue at once

GG_DEV unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Writes the finished sample's outcome and colour.  Runs once per ray, so it
// is kept out of line: its shading code (several pow) would otherwise sit in
// the hot stepping loop's instruction footprint.
__device__ __noinline__ void finish_sample(const DevParams& P, const DevOutputs& O, uint64_t idx,
                                           int cls, Ray R, uint32_t n_att, uint32_t n_acc,
                                           double intensity, double color_temp, bool crossed) {
  {
    const uint64_t n = P.n_rays;
    double lin[3];
    if (cls == kClsHorizon || cls == kClsBudget) {
      lin[0] = lin[1] = lin[2] = 0.0;
    } else if (cls == kClsEscaped) {
      if (P.sky == kSkyChecker)
        checker_sky(P, R.x[2], R.x[3], lin);
      else
        procedural_sky(R.v, lin);
    } else if (cls == kClsDisk) {
      disk_color(intensity, lin);
    } else {
      lin[0] = 0.0;
      lin[1] = 0.0;
      lin[2] = 10.0 / 255.0;
    }
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
  unsigned long long attempts, accepted, cls[5];
};

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

template <int METRIC, int DISK, int STEPPER>
__global__ void __launch_bounds__(kTraceBlock,
                                  METRIC == kMetricKerr ? kTraceMinBlocksKerr : kTraceMinBlocksSchw)
    trace_fp64_kernel(const __grid_constant__ DevParams P, const __grid_constant__ DevOutputs O,
                      DevControl* ctl) {
  const unsigned lane = threadIdx.x & 31u;
  __shared__ BlockStats bs;
  __shared__ double k_smem[7][4][kTraceBlock];  // stage derivatives, see KStore
  const KStore K{k_smem};
  if (threadIdx.x < sizeof(BlockStats) / 8)
    reinterpret_cast<unsigned long long*>(&bs)[threadIdx.x] = 0ull;
  __syncthreads();
  auto finish = [&](uint64_t i, int cls, const Ray& r, uint32_t na, uint32_t nc, double inten_o,
                    double temp_o, bool cr) {
    finish_sample(P, O, i, cls, r, na, nc, inten_o, temp_o, cr);
    atomicAdd(&bs.attempts, (unsigned long long)na);
    atomicAdd(&bs.accepted, (unsigned long long)nc);
    atomicAdd(&bs.cls[cls], 1ull);
  };

  Ray R;
  uint64_t idx = 0;
  bool live = false;
  uint32_t n_att = 0, n_acc = 0;
  double inten = 0.0, trans = 1.0;  // volumetric disk accumulators
  bool crossed = false;
  bool k1_valid = false;    // K(0, .) holds a(x, v) of the current state
  bool k7_pending = false;  // full DP: K(6, .) is the next k1, copy pending

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
          b = atomicAdd(&ctl->next_ray, (unsigned long long)kChunk);
          if (P.attempt_budget) {
            const unsigned long long used = atomicAdd(&ctl->budget_used, 0ull);
            if (used > P.attempt_budget) {
              atomicExch(&ctl->abort, 1u);
              b = P.n_rays;  // stop taking work
            }
          }
        }
        b = __shfl_sync(kFull, b, 0);
        if (b >= P.n_rays) {
          wdone = true;
          break;
        }
        wbase = b;
        const uint64_t left = P.n_rays - b;
        wcount = left < kChunk ? (uint32_t)left : kChunk;
      }
      const unsigned nn = (unsigned)__popc(need);
      const unsigned take = nn < wcount ? nn : wcount;
      const unsigned rank = (unsigned)__popc(need & lanemask_lt());
      if (!live && rank < take) {
        idx = wbase + rank;
        R = start_sample(P, idx);
        live = true;
        n_att = 0;
        n_acc = 0;
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
    for (int it = 0; it < kPeriod; ++it) {
      if (!live) continue;
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
        res = attempt_dp45_fp64<METRIC>(P, R, K, k1_valid, k7_pending, acc, h_used, end);
      else
        res = attempt_fp64<METRIC>(P, R, K, k1_valid, acc, h_used);
      n_att += 1;
      if (acc) n_acc += 1;
      int done_cls = -1;
      double out_int = 0.0, out_temp = 0.0;

      if (acc) {
        // The step's path: the reference's Euler segment (exactly linear in
        // the step fraction), or the full Dormand-Prince step's cubic Hermite.
        double raw[4];
#pragma unroll
        for (int i = 0; i < 4; ++i)
          raw[i] = STEPPER == kStepperDP45 ? end.xraw[i] : xb[i] + h_used * vb[i];
        auto point = [&](double s, double c[8]) {
          if (STEPPER == kStepperDP45) {
            double ka[4], kb[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
              kb[i] = K(0, i);
              ka[i] = K(6, i);
            }
            hermite_point(xb, vb, kb, raw, R.v, ka, h_used, s, c);
            normalize_coords(c);
          } else {
            segment_point(xb, vb, h_used, R.v, s, c);
          }
        };
        auto root = [&](int comp, double target, double linear_s) {
          return STEPPER == kStepperDP45 ? hermite_root(xb, vb, raw, R.v, h_used, comp, target)
                                         : linear_s;
        };
        // escape-sphere crossing on this step
        if (O.cross && xb[1] <= P.max_radius && raw[1] > P.max_radius) {
          double c[8];
          point(root(1, P.max_radius, (P.max_radius - xb[1]) / (raw[1] - xb[1])), c);
          store_cross(P, O, idx, c);
          crossed = true;
        }
        if (DISK == kDiskThin) {
          const double d_b = xb[2] - kHalfPi;
          const double d_a = R.x[2] - kHalfPi;
          if ((d_b < 0.0 && d_a >= 0.0) || (d_b > 0.0 && d_a <= 0.0)) {
            const double s = root(2, kHalfPi, d_b / (d_b - d_a));
            double c[8];
            point(s, c);
            const double r_c =
                STEPPER == kStepperDP45 ? c[1] : xb[1] + s * (raw[1] - xb[1]);
            if (r_c >= P.r_inner && r_c <= P.r_outer) {
              c[1] = r_c;
              c[2] = kHalfPi;
              const double g = redshift_factor<METRIC>(P, r_c, kHalfPi, c + 4);
              const double q = P.r_inner / r_c;
              const double g2 = g * g;
              out_int = (g2 * g2) * pow(q, P.emissivity_index);
              out_temp = g * pow(q, 0.75);
#pragma unroll
              for (int i = 0; i < 4; ++i) {
                R.x[i] = c[i];
                R.v[i] = c[4 + i];
              }
              R.lam = lam_b + s * h_used;
              store_cross(P, O, idx, c);
              crossed = true;
              done_cls = kClsDisk;
            }
          }
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
          if (!(cap_r < P.r_inner || cap_r > P.r_outer)) {
            const double qq = P.r_inner / cap_r;
            const double rho = P.density_0 * (qq * qq) *
                               exp(-z * z / (2.0 * P.scale_height * P.scale_height));
            if (rho > 0.0) {
              const double j = rho * rho * pow(qq, 0.75);
              double pm[4];
#pragma unroll
              for (int i = 0; i < 4; ++i) pm[i] = 0.5 * (vb[i] + R.v[i]);
              const double g = redshift_factor<METRIC>(P, mid[1], mid[2], pm);
              const double g2 = g * g;
              inten = inten + j * (g2 * g2) * dlambda * trans;
              trans = trans * exp(-rho * dlambda * 0.1);
              if (trans < 1e-3) {
                done_cls = kClsDisk;
                out_int = inten;
                out_temp = P.temperature_0;
              }
            }
          }
        }
        if (done_cls < 0 && res != kContinue) {
          if (inten > 0.0) {
            done_cls = kClsDisk;
            out_int = inten;
            out_temp = P.temperature_0;
          } else {
            done_cls = res == kEscaped ? kClsEscaped : kClsHorizon;
          }
        }
        if (done_cls < 0 && n_att >= P.max_steps) {
          if (inten > 0.0) {
            done_cls = kClsDisk;
            out_int = inten;
            out_temp = P.temperature_0;
          } else {
            done_cls = kClsMaxSteps;
          }
        }
      } else if (done_cls < 0) {
        if (res == kHorizon) done_cls = kClsHorizon;
        else if (res == kEscaped) done_cls = kClsEscaped;
        else if (n_att >= P.max_steps) done_cls = kClsMaxSteps;
      }
      if (done_cls >= 0) {
        finish(idx, done_cls, R, n_att, n_acc, out_int, out_temp, crossed);
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
          finish(idx, kClsBudget, R, n_att, n_acc, 0.0, 0.0, crossed);
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
#pragma unroll
    for (int k = 0; k < 5; ++k)
      if (bs.cls[k]) atomicAdd(&ctl->class_count[k], bs.cls[k]);
  }
}

// Averages the spp linear sample colours of each pixel in sample order and
// encodes sRGB (render_row, renderer.rs:326-343).
__global__ void reduce_samples_kernel(const __grid_constant__ DevParams P, const double* samples,
                                      uint8_t* rgb8) {
  const uint64_t n_pix = (uint64_t)P.width * P.height;
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

template <int METRIC, int DISK, int STEPPER>
const void* trace_fn() {
  return reinterpret_cast<const void*>(&trace_fp64_kernel<METRIC, DISK, STEPPER>);
}

template <int STEPPER>
const void* select_metric_disk(const DevParams& P) {
  if (P.metric == kMetricKerr) {
    if (P.disk == kDiskThin) return trace_fn<kMetricKerr, kDiskThin, STEPPER>();
    if (P.disk == kDiskVolumetric) return trace_fn<kMetricKerr, kDiskVolumetric, STEPPER>();
    return trace_fn<kMetricKerr, kDiskNone, STEPPER>();
  }
  if (P.disk == kDiskThin) return trace_fn<kMetricSchwarzschild, kDiskThin, STEPPER>();
  if (P.disk == kDiskVolumetric) return trace_fn<kMetricSchwarzschild, kDiskVolumetric, STEPPER>();
  return trace_fn<kMetricSchwarzschild, kDiskNone, STEPPER>();
}

const void* select_trace(const DevParams& P) {
  return P.stepper == kStepperDP45 ? select_metric_disk<kStepperDP45>(P)
                                   : select_metric_disk<kStepperReference>(P);
}

}  // namespace

cudaError_t trace_occupancy(const DevParams& P, int* blocks_per_sm) {
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, select_trace(P),
                                                       kTraceBlock, 0);
}

cudaError_t launch_trace(const DevParams& P, const DevOutputs& O, DevControl* ctl, int grid,
                         cudaStream_t stream) {
  const void* fn = select_trace(P);
  DevParams p = P;
  DevOutputs o = O;
  void* args[] = {&p, &o, &ctl};
  return cudaLaunchKernel(fn, dim3(grid), dim3(kTraceBlock), args, 0, stream);
}

cudaError_t launch_reduce(const DevParams& P, const double* samples, uint8_t* rgb8, int sms,
                          cudaStream_t stream) {
  const uint64_t n_pix = (uint64_t)P.width * P.height;
  uint64_t blocks = (n_pix + 255) / 256;
  const uint64_t cap = (uint64_t)sms * 8;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  reduce_samples_kernel<<<(unsigned)blocks, 256, 0, stream>>>(P, samples, rgb8);
  return cudaGetLastError();
}

}  // namespace gg
