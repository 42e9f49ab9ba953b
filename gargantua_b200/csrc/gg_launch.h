// gg_launch.h -- host-side launch entry points of the trace kernels.
#pragma once

#include <cuda_runtime.h>

#include "gg_params.h"

namespace gg {

#ifndef GG_TRACE_MIN_BLOCKS
#define GG_TRACE_MIN_BLOCKS 4
#endif

constexpr int kTraceBlock = 128;  // threads per CTA of the trace kernels
// resident CTAs per SM the register budget targets (65536 / (128 * 4) = 128
// registers; the few spills this forces cost less than the extra warps gain)
constexpr int kTraceMinBlocks = GG_TRACE_MIN_BLOCKS;

// Resident CTAs per SM of the trace kernel `P` selects.
cudaError_t trace_occupancy(const DevParams& P, int* blocks_per_sm);

// Persistent trace over P.n_rays samples; `grid` CTAs of kTraceBlock threads.
cudaError_t launch_trace(const DevParams& P, const DevOutputs& O, DevControl* ctl, int grid,
                         cudaStream_t stream);

// Best-of-5 FMA throughput (FLOP/s, FMA = 2) of the current device.
cudaError_t measure_fma_peak(int fp64, int sms, double* flops);

// Per-pixel average of spp linear sample colours + sRGB encode.
cudaError_t launch_reduce(const DevParams& P, const double* samples, uint8_t* rgb8, int sms,
                          cudaStream_t stream);

}  // namespace gg
