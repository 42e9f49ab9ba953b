// gg_launch.h -- host-side launch entry points of the trace kernels.
#pragma once

#include <cuda_runtime.h>

#include "gg_params.h"

namespace gg {

constexpr int kTraceBlock = 128;  // threads per CTA of the trace kernels

// Resident CTAs per SM of the trace kernel `P` selects.
cudaError_t trace_occupancy(const DevParams& P, int* blocks_per_sm);

// Persistent trace over P.n_rays samples; `grid` CTAs of kTraceBlock threads.
cudaError_t launch_trace(const DevParams& P, const DevOutputs& O, DevControl* ctl, int grid,
                         cudaStream_t stream);

// Per-pixel average of spp linear sample colours + sRGB encode.
cudaError_t launch_reduce(const DevParams& P, const double* samples, uint8_t* rgb8, int sms,
                          cudaStream_t stream);

}  // namespace gg
