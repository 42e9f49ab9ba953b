// gg_launch.h -- host-side launch entry points of the trace kernels.
#pragma once

#include <cuda_runtime.h>

#include "gg_params.h"

namespace gg {

constexpr int kTraceBlock = 128;  // threads per CTA of the trace kernels

// Resident CTAs per SM each metric's trace kernel is register-budgeted for
// (65536 / (128 * blocks) registers per thread).  Kerr's stepping loop hides
// FP64 latency better with 6 CTAs (80 registers, k vectors in shared
// memory) despite a few spills; Schwarzschild's lighter right-hand side is
// fastest at 4.  Measured on B200, Kerr 1920x1080: 4 -> 53.8 ms, 5 -> 50.9
// ms, 6 -> 49.2 ms.  GG_TRACE_MIN_BLOCKS overrides both (tuning builds).
#ifdef GG_TRACE_MIN_BLOCKS
constexpr int kTraceMinBlocksKerr = GG_TRACE_MIN_BLOCKS;
constexpr int kTraceMinBlocksSchw = GG_TRACE_MIN_BLOCKS;
#else
constexpr int kTraceMinBlocksKerr = 6;
constexpr int kTraceMinBlocksSchw = 4;
#endif

// Resident CTAs per SM the mixed-precision trace kernel is budgeted for.
#ifdef GG_MIXED_MIN_BLOCKS
constexpr int kMixedMinBlocks = GG_MIXED_MIN_BLOCKS;
#else
constexpr int kMixedMinBlocks = 8;
#endif

// Resident CTAs per SM of the trace kernel `P` selects.
cudaError_t trace_occupancy(const DevParams& P, int* blocks_per_sm);

// Persistent trace over P.n_rays samples; `grid` CTAs of kTraceBlock threads.
cudaError_t launch_trace(const DevParams& P, const DevOutputs& O, DevControl* ctl, int grid,
                         cudaStream_t stream);

// Mixed form (P.precision == GG_PREC_MIXED, full Dormand-Prince): the FP32
// pass over the samples, which hands FP64-band rays to O.queue, and the FP64
// pass over that queue, which (P.hand_back) returns rays clear of the band to
// O.ret; then, after launch_next_round, the FP32 pass over O.ret (`returned`)
// and a last FP64 pass without hand-back.
// A batched render (batch != nullptr) runs one of kBatchVariants kernel
// variants (compaction period x register budget), chosen by `variant`.
constexpr int kBatchVariants = 6;
cudaError_t mixed_occupancy(const DevParams& P, int* blocks_per_sm,
                            const BatchTable* batch = nullptr, int variant = 0,
                            bool returned = false);
cudaError_t launch_mixed(const DevParams& P, const DevOutputs& O, DevControl* ctl, int grid,
                         cudaStream_t stream, const BatchTable* batch = nullptr,
                         int variant = 0, bool returned = false);
cudaError_t launch_next_round(DevControl* ctl, cudaStream_t stream);
cudaError_t queue_trace_occupancy(const DevParams& P, int* blocks_per_sm);
cudaError_t launch_queue_trace(const DevParams& P, const DevOutputs& O, DevControl* ctl,
                               int grid, cudaStream_t stream,
                               const BatchTable* batch = nullptr);

// Differentiable render: the adjoint pass (gg_adjoint.cu) of a forward run
// by launch_trace with P.ckpt set; grad5 (device) accumulates dL/d(a,
// inclination, r_cam, r_inner, q).
// list_buf (device, backward_list_bytes) holds the pass's sorted work list.
size_t backward_list_bytes(uint64_t n_rays, uint32_t n_keys);
cudaError_t launch_diff_backward(const DevParams& P, const DiffOut& D, const double* dl_drgb,
                                 double* grad5, void* list_buf, int sms, cudaStream_t stream);

// Best-of-5 FMA throughput (FLOP/s, FMA = 2) of the current device.
cudaError_t measure_fma_peak(int fp64, int sms, double* flops);

// Per-pixel average of spp linear sample colours + sRGB encode.
cudaError_t launch_reduce(const DevParams& P, const double* samples, uint8_t* rgb8, int sms,
                          cudaStream_t stream);

}  // namespace gg
