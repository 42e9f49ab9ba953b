// gg_launch.h -- host-side launch entry points of the trace kernels.
#pragma once

#include <cuda_runtime.h>

#include "gg_params.h"

namespace gg {

constexpr int kTraceBlock = 128;  // threads per CTA of the trace kernels

// Resident CTAs per SM the FP64 trace kernel is register-budgeted for
// (65536 / (128 * blocks) registers per thread).  Kerr camera passes: 5 (102
// registers); Kerr passes set by their longest ray chains -- the mixed form's
// FP64 band passes, the differentiable render's forward, camera passes of
// fewer than 2^20 samples -- 4 (128 registers, no spills on the chain);
// Schwarzschild's lighter right-hand side: 4.
// Measured on B200 (ms, CTAs 6 / 5 / 4): FP64 drop-in Kerr 1080p 45.3 /
// 43.8 / 44.8, its full Dormand-Prince form 59.4 / 55.3 / 55.4, the stress
// frame at 2048^2 x 4 spp 133.5 / 133.6 / 136.2 (drop-in) and 171.7 / 160.4
// / 161.9 (full DP); band passes, through the mixed 1080p frame 27.0 / 26.7 /
// 26.3; the 512^2 adjoint's forward 10.1 / 8.9 / 8.6.  At 3 CTAs (168
// registers) for the band passes and the mixed pass over returned rays, the
// 1080p frame gains 0.3 ms but the stress frame at 2048^2 x 4 spp, whose band
// holds 12 % of the attempts, loses 1.3 ms.  The camera passes' budget (5)
// for the band passes of renders from 2^23 samples, whose band holds enough
// rays to be throughput-bound: 84.9 against 84.2 ms on the stress frame at
// 2048^2 x 4 spp, 1.291 against 1.285 s at 4096^2 x 16 spp and 2.403 against
// 2.385 s on the 2,048-scene batch, so not kept.  GG_TRACE_MIN_BLOCKS overrides
// all three, GG_TRACE_CHAIN_MIN_BLOCKS the chain-bound one (tuning builds).
#ifdef GG_TRACE_MIN_BLOCKS
constexpr int kTraceMinBlocksKerr = GG_TRACE_MIN_BLOCKS;
constexpr int kTraceMinBlocksKerrChain = GG_TRACE_MIN_BLOCKS;
constexpr int kTraceMinBlocksSchw = GG_TRACE_MIN_BLOCKS;
#else
constexpr int kTraceMinBlocksKerr = 5;
#ifdef GG_TRACE_CHAIN_MIN_BLOCKS
constexpr int kTraceMinBlocksKerrChain = GG_TRACE_CHAIN_MIN_BLOCKS;
#else
constexpr int kTraceMinBlocksKerrChain = 4;
#endif
constexpr int kTraceMinBlocksSchw = 4;
#endif

// Resident CTAs per SM the mixed-precision trace kernel is budgeted for: its
// camera pass (8, 64 registers: throughput), and its pass over the rays the
// FP64 pass hands back (4, 128 registers: set by its longest ray chains).
// Measured on the 1080p Kerr frame (ms; camera / returned CTAs): 8 / 8 26.4,
// 7 / 7 26.1, 6 / 6 26.6, 8 / 6 25.9, 8 / 4 25.5, 7 / 4 25.6.
#ifdef GG_MIXED_MIN_BLOCKS
constexpr int kMixedMinBlocks = GG_MIXED_MIN_BLOCKS;
#else
constexpr int kMixedMinBlocks = 8;
#endif
#ifdef GG_MIXED_RET_MIN_BLOCKS
constexpr int kMixedMinBlocksReturned = GG_MIXED_RET_MIN_BLOCKS;
#else
constexpr int kMixedMinBlocksReturned = 4;
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
struct BatchVariant {
  int period, ctas_per_sm, block, chunk;
};
// Refill period, CTAs per SM (the register budget: 65536 / (block * CTAs)
// per thread), threads per CTA and samples a warp claims per queue access.
constexpr BatchVariant kBatchVariantTable[] = {
    {16, 8, 128, 32}, {8, 8, 128, 32},  {4, 8, 128, 32},  {16, 7, 128, 32},
    {32, 7, 128, 32}, {32, 8, 128, 32}, {32, 16, 64, 32}, {16, 16, 64, 32},
    {32, 4, 256, 32}, {16, 4, 256, 32}, {32, 8, 128, 16}, {32, 8, 128, 64}};
constexpr int kBatchVariants = (int)(sizeof(kBatchVariantTable) / sizeof(kBatchVariantTable[0]));
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
