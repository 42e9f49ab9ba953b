// gg_peak.cu -- FP64 / FP32 FMA throughput probe (the ALU roofline's peak).
//
// The trace kernels are bound by the FP64 (plain form) or FP32 (mixed form)
// FMA pipes, not by HBM or tensor cores, so their roofline denominator is the
// chip's FMA throughput measured on this device: every thread runs eight
// independent FMA chains for a fixed number of iterations (no loads in the
// loop; one store per thread at the end so the work cannot be elided).
#include <cuda_runtime.h>

#include <cstdint>

#include "gg_launch.h"

namespace gg {

namespace {

constexpr int kChains = 8;

template <class T>
__global__ void __launch_bounds__(256) fma_chains_kernel(T* sink, int iters, T b, T c) {
  T a[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k) a[k] = T(threadIdx.x + k) * T(1e-3);
#pragma unroll 1
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int r = 0; r < 16; ++r) {
#pragma unroll
      for (int k = 0; k < kChains; ++k) a[k] = fma(a[k], b, c);
    }
  }
  T s = T(0);
#pragma unroll
  for (int k = 0; k < kChains; ++k) s += a[k];
  sink[(uint64_t)blockIdx.x * blockDim.x + threadIdx.x] = s;
}

template <class T>
cudaError_t run(int sms, int iters, int reps, double* best_flops) {
  const int blocks = sms * 8, threads = 256;
  T* sink = nullptr;
  cudaError_t e = cudaMalloc(&sink, sizeof(T) * (size_t)blocks * threads);
  if (e != cudaSuccess) return e;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  double best = 0.0;
  for (int r = 0; r < reps + 1 && e == cudaSuccess; ++r) {
    cudaEventRecord(a);
    fma_chains_kernel<T><<<blocks, threads>>>(sink, iters, T(0.999999), T(1e-7));
    cudaEventRecord(b);
    e = cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    const double flops = 2.0 * kChains * 16.0 * iters * (double)blocks * threads;
    if (r > 0 && ms > 0.f && flops / (ms * 1e-3) > best) best = flops / (ms * 1e-3);
  }
  if (e == cudaSuccess) e = cudaGetLastError();
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(sink);
  *best_flops = best;
  return e;
}

}  // namespace

cudaError_t measure_fma_peak(int fp64, int sms, double* flops) {
  return fp64 ? run<double>(sms, 2048, 5, flops) : run<float>(sms, 4096, 5, flops);
}

}  // namespace gg
