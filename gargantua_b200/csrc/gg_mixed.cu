// gg_mixed.cu -- the mixed-precision persistent trace kernel (GG_PREC_MIXED).
//
// Same work decomposition as the FP64 kernel (gg_trace.cu): persistent CTAs,
// 32-sample chunks per warp, ballot refill every PERIOD attempts.  Each lane
// steps its ray with the mixed-precision full Dormand-Prince attempt
// (gg_mixed.cuh).  When a ray's next attempt would start inside the FP64
// band -- r within 0.5 M of the horizon (with its buffer) or of the prograde
// photon orbit, theta within pole_band of a pole, or a step that would carry
// theta across a pole -- the lane writes the ray's state, in FP64, to a
// global queue and takes a new sample.  The FP64 kernel then runs over that
// queue in a second launch (trace_fp64_kernel<..., kSrcQueue>), which, in
// renders of 2^20 samples or more, hands rays that leave the band back to a
// return queue; this kernel continues those (SRC = kSrcQueue) in a third
// launch, and a last FP64 launch finishes the rays that re-entered the band.
// Handing rays off instead of running FP64 attempts inside this kernel keeps
// every launch warp-uniform: a warp never executes the FP32 and the FP64
// attempt back to back for lanes in different bands.
//
// Crossings of the escape sphere and the disk plane are detected on the
// float-pair differences and located in FP64 on the step's continuous
// extension (the Dormand-Prince dense output), as in the FP64 kernel.
#include <cuda_runtime.h>

#include <cstdint>
#include <utility>

#include "../../include/gargantua_gpu.h"
#include "gg_device.cuh"
#include "gg_launch.h"
#include "gg_mixed.cuh"
#include "gg_trace_common.cuh"

namespace gg {

namespace {

// Writes the ray to the FP64 pass's queue (out of line: once per handed-off
// ray).  The state is the one the next attempt starts from.  The register
// part of the ray comes by value, so the stepping loop keeps it in registers.
template <class KS>
__device__ __noinline__ void hand_off(const DevOutputs& O, DevControl* ctl, KS K,
                                      MixedRegs S, uint32_t n_att, uint32_t n_acc,
                                      uint32_t scene) {
  const unsigned long long slot = atomicAdd(&ctl->queued, 1ull);
  if (slot >= O.queue_cap) {
    atomicExch(&ctl->queue_overflow, 1u);
    return;
  }
  const Ray R = mixed_fp64(K, S);
  QueuedRay& q = O.queue[slot];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    q.x[i] = R.x[i];
    q.v[i] = R.v[i];
  }
  q.h = R.h;
  q.lam = R.lam;
  q.idx = K.idx();
  q.n_att = n_att;
  q.n_acc = n_acc;
  q.scene = scene;
}

// Scene of global sample g in a batched launch: the last k with first[k] <= g.
GG_DEV uint32_t find_scene(const BatchTable& B, uint64_t g) {
  uint32_t lo = 0, hi = B.n;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (B.first[mid] <= g) lo = mid; else hi = mid;
  }
  return lo;
}

// Writes a finished ray's outcome (its state converted to FP64) and counts it
// in the block's statistics.  Out of line, once per ray.
template <class KS>
__device__ __noinline__ void mixed_finish(const DevParams& P, const DevOutputs& O, KS K,
                                          MixedRegs S, int cls, uint32_t n_att, uint32_t n_acc,
                                          bool crossed, BlockStats* bs) {
  const Ray R = mixed_fp64(K, S);
  finish_sample(P, O, K.idx(), cls, R, n_att, n_acc, 0.0, 0.0, crossed, R.x[2], R.x[3]);
  atomicAdd(&bs->attempts, (unsigned long long)n_att);
  atomicAdd(&bs->accepted, (unsigned long long)n_acc);
  atomicAdd(&bs->cls[cls], 1ull);
}

// An accepted step's data for its continuous extension, read where it lives:
// the pre-step state in FP64 (B), the increments and the seven stage
// derivatives in this lane's shared-memory column (no step record in local
// memory).
template <class KS>
struct MixedSpan {
  KS K;
  Ray B;
  double h;
  GG_DEV double xb(int c) const { return B.x[c]; }
  GG_DEV double vb(int c) const { return B.v[c]; }
  GG_DEV double xa(int c) const { return B.x[c] + (double)K.comp(kSlotDx, c); }
  GG_DEV double va(int c) const { return B.v[c] + (double)K.comp(kSlotDv, c); }
  GG_DEV double k(int l, int c) const { return (double)K.comp(l, c); }
};

// The accepted step (pre-step state, increments in slots 7, 8, k1 in slot
// 0, k7 in slot 6) crossed the escape sphere (`esc`) and/or the disk
// plane (`dsk`): locate the crossings in FP64 on the step's continuous
// extension.
// Stores the escape crossing.  When the ray ends here -- on the thin disk,
// or, with the checkerboard sky, at the escape sphere (whose cell is read at
// the crossing; the next attempt would only find r > max_radius and return
// Escaped, and is counted) -- writes its outcome and returns the attempts it
// ended with, else 0.
template <int METRIC, int DISK, class KS>
__device__ __noinline__ uint32_t mixed_crossings(const DevParams& P, const DevOutputs& O, KS K,
                                             MixedRegs S, float hf, bool esc, bool dsk,
                                             uint32_t n_att, uint32_t n_acc, BlockStats* bs) {
  const Ray B = mixed_fp64(K, S);
  const uint64_t idx = K.idx();
  const MixedSpan<KS> sp{K, B, (double)hf};
  bool esc_end = false;
  double sky_th = 0.0, sky_ph = 0.0;
  if (esc && (O.cross || P.sky == kSkyChecker)) {
    double c[8];
    dense_crossing_src<1>(sp, P.max_radius, c);
    normalize_coords(c);
    if (O.cross) store_cross(P, O, idx, c);
    esc_end = P.sky == kSkyChecker;
    sky_th = c[2];
    sky_ph = c[3];
  }
  if (DISK == kDiskThin && dsk) {
    double c[8];
    const double s = dense_crossing_src<2>(sp, kHalfPi, c);
    normalize_coords(c);
    const double r_c = c[1];
    if (r_c >= P.r_inner && r_c <= P.r_outer) {
      c[2] = kHalfPi;
      const double g = redshift_factor<METRIC>(P, r_c, kHalfPi, c + 4);
      const double q = P.r_inner / r_c;
      const double g2 = g * g;
      Ray end;
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        end.x[i] = c[i];
        end.v[i] = c[4 + i];
      }
      end.h = S.h;
      end.lam = B.lam + s * sp.h;
      store_cross(P, O, idx, c);
      finish_sample(P, O, idx, kClsDisk, end, n_att, n_acc, (g2 * g2) * pow(q, P.emissivity_index),
                    g * pow(q, 0.75), true, c[2], c[3]);
      atomicAdd(&bs->attempts, (unsigned long long)n_att);
      atomicAdd(&bs->accepted, (unsigned long long)n_acc);
      atomicAdd(&bs->cls[kClsDisk], 1ull);
      return n_att;
    }
  }
  if (esc_end && n_att < P.max_steps) {
    Ray end;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      end.x[i] = sp.xa(i);
      end.v[i] = sp.va(i);
    }
    normalize_coords(end.x);
    end.h = S.h;
    end.lam = B.lam + sp.h;
    const uint32_t na = n_att + 1;
    finish_sample(P, O, idx, kClsEscaped, end, na, n_acc, 0.0, 0.0, true, sky_th, sky_ph);
    atomicAdd(&bs->attempts, (unsigned long long)na);
    atomicAdd(&bs->accepted, (unsigned long long)n_acc);
    atomicAdd(&bs->cls[kClsEscaped], 1ull);
    return na;
  }
  return 0;
}

// Deferred per-ray work of a lane (low bits) and its flags.
constexpr uint32_t kPendHandOff = 1, kPendCross = 2, kPendFinish = 3, kPendKind = 0xf;
constexpr uint32_t kPendEsc = 0x10, kPendDsk = 0x20;  // kPendCross: which crossings
constexpr uint32_t kPendClsShift = 8;                  // kPendFinish: the class

// BUDGET: the render has an attempt budget (its bookkeeping costs registers,
// so renders without one run a variant that has none).  BATCH: the samples
// are the concatenated samples of many scenes (B); each lane looks up its
// sample's scene, whose parameters and outputs replace P and O for that ray
// (the integrator, sky kind and budget are the batch's, in P).  PERIOD
// (attempts between refills) and MINB (CTAs per SM the registers are
// budgeted for) are the settings the batch autotuner chooses between.
// SRC: kSrcCamera starts the samples from the camera; kSrcQueue continues the
// rays the FP64 pass handed back (O.ret, ctl->returned of them).  BLOCK
// (threads per CTA) and CHUNK (samples a warp claims from the work queue at
// a time) are the batch autotuner's other two settings.  The CTA's column
// (mixed_smem_bytes<BLOCK>) is dynamic shared memory.
template <int METRIC, int DISK, bool BUDGET, bool BATCH, int PERIOD, int MINB, int SRC,
          int BLOCK = kTraceBlock, int CHUNK = (int)kChunk>
__global__ void __launch_bounds__(BLOCK, MINB)
    trace_mixed_kernel(const __grid_constant__ DevParams P, const __grid_constant__ DevOutputs O,
                       DevControl* ctl, const __grid_constant__ BatchTable B) {
  const unsigned lane = threadIdx.x & 31u;
  __shared__ BlockStats bs;
  extern __shared__ __align__(16) unsigned char mixed_smem[];
  const MixedSmemT<BLOCK> K = MixedSmemT<BLOCK>::at(mixed_smem);
  if (threadIdx.x < sizeof(BlockStats) / 8)
    reinterpret_cast<unsigned long long*>(&bs)[threadIdx.x] = 0ull;
  __syncthreads();

  MixedRegs S;
  uint32_t scene = 0;  // BATCH: the ray's scene
  bool live = false;
  uint32_t n_att = 0, n_acc = 0;
  bool crossed = false;
  bool k1_valid = false;
  bool k7_pending = false;
  // Per-ray work found during the attempts (hand-off, crossing, finish) is
  // deferred to the top of the loop, where every lane of the warp that has
  // some runs it together instead of one lane at a time mid-period.
  uint32_t pend = 0;      // kPend* | flags
  float pend_hf = 0.0f;   // kPendCross: the accepted step awaiting its crossing

  uint64_t wbase = 0;
  uint32_t wcount = 0;
  bool wdone = false;
  unsigned budget_pending = 0;
  const uint64_t n_src =
      SRC == kSrcQueue ? (ctl->returned < O.ret_cap ? ctl->returned : O.ret_cap) : P.n_rays;
  unsigned long long* const head = SRC == kSrcQueue ? &ctl->next_returned : &ctl->next_ray;

  for (;;) {
    // ---- deferred per-ray work ---------------------------------------------
    if (pend) {
      const DevParams& PL = BATCH ? B.scenes[scene].P : P;
      const DevOutputs& OL = BATCH ? B.scenes[scene].O : O;
      const uint32_t kind = pend & kPendKind;
      if (kind == kPendHandOff) {
        hand_off(O, ctl, K, S, n_att, n_acc, scene);
      } else if (kind == kPendCross) {
        const uint32_t ended = mixed_crossings<METRIC, DISK>(
            PL, OL, K, S, pend_hf, (pend & kPendEsc) != 0, (pend & kPendDsk) != 0, n_att, n_acc, &bs);
        if (ended) {
          if (BUDGET) budget_pending += ended;
        } else {
          mixed_advance(S, K, pend_hf, k1_valid, k7_pending);
          if (n_att >= PL.max_steps) {
            mixed_finish(PL, OL, K, S, kClsMaxSteps, n_att, n_acc, crossed, &bs);
            if (BUDGET) budget_pending += n_att;
          } else {
            live = true;
          }
        }
      } else {
        mixed_finish(PL, OL, K, S, (int)(pend >> kPendClsShift), n_att, n_acc, crossed, &bs);
        if (BUDGET) budget_pending += n_att;
      }
      pend = 0;
    }

    // ---- refill lanes whose ray finished or was handed off ----------------
    unsigned need = __ballot_sync(kFull, !live);
    if (BUDGET && need && !wdone) {
      unsigned long long ab = 0;
      if (lane == 0) ab = atomicOr(&ctl->abort, 0u);
      if (__shfl_sync(kFull, ab, 0)) wdone = true;
    }
    while (need && !wdone) {
      if (wcount == 0) {
        unsigned long long b = 0;
        if (lane == 0) {
          b = atomicAdd(head, (unsigned long long)CHUNK);
          if (BUDGET) {
            const unsigned long long used = atomicAdd(&ctl->budget_used, 0ull);
            if (used > P.attempt_budget) {
              atomicExch(&ctl->abort, 1u);
              b = n_src;
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
        wcount = left < (uint64_t)CHUNK ? (uint32_t)left : (uint32_t)CHUNK;
      }
      const unsigned nn = (unsigned)__popc(need);
      const unsigned take = nn < wcount ? nn : wcount;
      const unsigned rank = (unsigned)__popc(need & lanemask_lt());
      if (!live && rank < take) {
        if (SRC == kSrcQueue) {
          const QueuedRay& q = O.ret[wbase + rank];
          Ray R;
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            R.x[i] = q.x[i];
            R.v[i] = q.v[i];
          }
          R.h = q.h;
          R.lam = q.lam;
          if (BATCH) scene = q.scene;
          mixed_load(R, q.idx, K, S);
          n_att = q.n_att;
          n_acc = q.n_acc;
        } else {
          uint64_t idx = BATCH ? wbase + rank : camera_sample(P, wbase + rank);
          if (BATCH) {
            scene = find_scene(B, idx);
            idx -= B.first[scene];
          }
          mixed_load(start_sample(BATCH ? B.scenes[scene].P : P, idx), idx, K, S);
          n_att = 0;
          n_acc = 0;
        }
        live = true;
        crossed = false;
        k1_valid = false;
        k7_pending = false;
      }
      wbase += take;
      wcount -= take;
      need = __ballot_sync(kFull, !live);
    }
    if (!__any_sync(kFull, live)) break;

    // ---- advance every live ray by up to PERIOD attempts ------------------
#pragma unroll 1
    for (int it = 0; it < PERIOD; ++it) {
      if (!live) continue;
      const DevParams& PL = BATCH ? B.scenes[scene].P : P;
      {
        const float r = K.comp(kSlotXh, 1), th = K.comp(kSlotXh, 2);
        if (r < PL.band_r || th < PL.pole_band || th > kPiHi - PL.pole_band) {
          pend = kPendHandOff;
          live = false;
          continue;
        }
      }
      bool acc;
      float hf = 0.0f;
      const int res = attempt_dp45_mixed<METRIC>(PL, S, K, k1_valid, k7_pending, acc, hf);
      n_att += 1;
      if (acc) {
        const float4 dx = K.get(kSlotDx);
        const float xh_r = K.comp(kSlotXh, 1), xh_th = K.comp(kSlotXh, 2);
        const float th_a = xh_th + dx.z;
        if (!(th_a > 0.0f && th_a < kPiHi)) {
          // theta would turn through a pole: re-take this step in FP64
          n_att -= 1;
          pend = kPendHandOff;
          live = false;
          continue;
        }
        n_acc += 1;
        const float dr_b = ff_minus(xh_r, K.comp(kSlotXl, 1), PL.max_radius_hi, PL.max_radius_lo);
        const bool esc = dr_b <= 0.0f && dr_b + dx.y > 0.0f;
        bool dsk = false;
        if (DISK == kDiskThin) {
          const float d_b = ff_minus(xh_th, K.comp(kSlotXl, 2), kHalfPiHi, kHalfPiLo);
          const float d_a = d_b + dx.z;
          dsk = (d_b < 0.0f && d_a >= 0.0f) || (d_b > 0.0f && d_a <= 0.0f);
        }
        if (esc || dsk) {
          if (esc && O.cross) crossed = true;
          pend = kPendCross | (esc ? kPendEsc : 0u) | (dsk ? kPendDsk : 0u);
          pend_hf = hf;
          live = false;
          continue;
        }
        mixed_advance(S, K, hf, k1_valid, k7_pending);
      }
      if (res == kEscaped || n_att >= PL.max_steps) {
        pend = kPendFinish | ((uint32_t)(res == kEscaped ? kClsEscaped : kClsMaxSteps)
                              << kPendClsShift);
        live = false;
      }
    }
    if (BUDGET) {
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
          mixed_finish(BATCH ? B.scenes[scene].P : P, BATCH ? B.scenes[scene].O : O, K, S,
                       kClsBudget, n_att, n_acc, crossed, &bs);
          live = false;
        }
      }
    }
  }

  __syncthreads();
  if (threadIdx.x == 0) {
    atomicAdd(&ctl->attempts, bs.attempts);
    atomicAdd(&ctl->accepted, bs.accepted);
#pragma unroll
    for (int k = 0; k < kNumClasses; ++k)
      if (bs.cls[k]) atomicAdd(&ctl->class_count[k], bs.cls[k]);
  }
}

// A kernel of the mixed form with its block size and dynamic shared memory.
struct MixedKernel {
  const void* fn;
  int block;
  int smem;
};

template <int METRIC, int DISK, bool BUDGET, bool BATCH = false, int PERIOD = kMixedPeriod,
          int MINB = kMixedMinBlocks, int SRC = kSrcCamera, int BLOCK = kTraceBlock,
          int CHUNK = (int)kChunk>
MixedKernel mixed_fn() {
  return {reinterpret_cast<const void*>(
              &trace_mixed_kernel<METRIC, DISK, BUDGET, BATCH, PERIOD, MINB, SRC, BLOCK, CHUNK>),
          BLOCK, mixed_smem_bytes<BLOCK>()};
}

template <bool BUDGET>
MixedKernel select_mixed_disk(const DevParams& P) {
  if (P.metric == kMetricKerr)
    return P.disk == kDiskThin ? mixed_fn<kMetricKerr, kDiskThin, BUDGET>()
                               : mixed_fn<kMetricKerr, kDiskNone, BUDGET>();
  return P.disk == kDiskThin ? mixed_fn<kMetricSchwarzschild, kDiskThin, BUDGET>()
                             : mixed_fn<kMetricSchwarzschild, kDiskNone, BUDGET>();
}

// The pass over the rays the FP64 pass handed back (no attempt budget: the
// hand-back is off in budgeted renders).
template <bool BATCH>
MixedKernel select_returned(const DevParams& P) {
  constexpr int Pd = kMixedPeriod, Mb = kMixedMinBlocksReturned;
  if (P.metric == kMetricKerr)
    return P.disk == kDiskThin
               ? mixed_fn<kMetricKerr, kDiskThin, false, BATCH, Pd, Mb, kSrcQueue>()
               : mixed_fn<kMetricKerr, kDiskNone, false, BATCH, Pd, Mb, kSrcQueue>();
  return P.disk == kDiskThin
             ? mixed_fn<kMetricSchwarzschild, kDiskThin, false, BATCH, Pd, Mb, kSrcQueue>()
             : mixed_fn<kMetricSchwarzschild, kDiskNone, false, BATCH, Pd, Mb, kSrcQueue>();
}

// Batched launches: variant v of kBatchVariantTable (refill period, CTAs per
// SM the registers are budgeted for, threads per CTA, samples per queue
// claim); the metric and disk kind are the batch's.
template <int METRIC, int DISK, int V>
MixedKernel batch_v() {
  constexpr BatchVariant b = kBatchVariantTable[V];
  return mixed_fn<METRIC, DISK, false, true, b.period, b.ctas_per_sm, kSrcCamera, b.block,
                  b.chunk>();
}

template <int METRIC, int DISK, int... Vs>
MixedKernel batch_variant(int v, std::integer_sequence<int, Vs...>) {
  MixedKernel k{nullptr, 0, 0};
  ((v == Vs ? (k = batch_v<METRIC, DISK, Vs>(), 0) : 0), ...);
  return k.fn ? k : batch_v<METRIC, DISK, 0>();
}

MixedKernel select_batch(const DevParams& P, int v) {
  const auto all = std::make_integer_sequence<int, kBatchVariants>{};
  if (P.metric == kMetricKerr)
    return P.disk == kDiskThin ? batch_variant<kMetricKerr, kDiskThin>(v, all)
                               : batch_variant<kMetricKerr, kDiskNone>(v, all);
  return P.disk == kDiskThin ? batch_variant<kMetricSchwarzschild, kDiskThin>(v, all)
                             : batch_variant<kMetricSchwarzschild, kDiskNone>(v, all);
}

MixedKernel select_kernel(const DevParams& P, const BatchTable* batch, int variant,
                          bool returned) {
  if (returned) return batch ? select_returned<true>(P) : select_returned<false>(P);
  if (batch) return select_batch(P, variant);
  return P.attempt_budget ? select_mixed_disk<true>(P) : select_mixed_disk<false>(P);
}

}  // namespace

cudaError_t mixed_occupancy(const DevParams& P, int* blocks_per_sm, const BatchTable* batch,
                            int variant, bool returned) {
  const MixedKernel k = select_kernel(P, batch, variant, returned);
  // opts in to more than 48 KB of dynamic shared memory where a variant
  // needs it (idempotent; launches follow an occupancy query)
  const cudaError_t e =
      cudaFuncSetAttribute(k.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, k.smem);
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k.fn, k.block, k.smem);
}

cudaError_t launch_mixed(const DevParams& P, const DevOutputs& O, DevControl* ctl, int grid,
                         cudaStream_t stream, const BatchTable* batch, int variant,
                         bool returned) {
  const MixedKernel k = select_kernel(P, batch, variant, returned);
  DevParams p = P;
  DevOutputs o = O;
  BatchTable b{};
  if (batch) b = *batch;
  void* args[] = {&p, &o, &ctl, &b};
  return cudaLaunchKernel(k.fn, dim3(grid), dim3(k.block), args, k.smem, stream);
}

}  // namespace gg

// The mixed kernel's polar-angle sincos evaluated on the host from the same
// source, so tests can check it against a double-precision reference.
extern "C" GG_API int gg_polar_sincos(const float* theta, float* s, float* c, uint32_t n) {
  if (!theta || !s || !c) return -1;
  for (uint32_t i = 0; i < n; ++i) gg::sincos_polar(theta[i], s + i, c + i);
  return 0;
}
