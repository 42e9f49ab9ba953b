// gg_checks.cu -- device functions of the ray path exported one by one, so
// that tests can compare them bit for bit with the oracle on identical
// inputs.  No counterpart in the reference; not used by any render.
//
// The starfield (sky.rs:26-40) hashes the f64 bits of a ray's final
// direction, so a one-ulp difference anywhere before it moves a star.  A
// full-frame comparison only shows that the two sides agree where their
// directions agree; these entries feed the device code and the oracle the
// same directions (and the same velocities for spatial_dir) instead.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/gargantua_gpu.h"
#include "gg_device.cuh"
#include "gg_mixed.cuh"
#include "gg_vjp.cuh"

namespace {

__global__ void sky_dir_kernel(const double* __restrict__ dirs, double* __restrict__ rgb,
                               uint64_t n) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    double c[3];
    gg::procedural_sky_dir(dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2], c);
    rgb[3 * i] = c[0];
    rgb[3 * i + 1] = c[1];
    rgb[3 * i + 2] = c[2];
  }
}

__global__ void spatial_dir_kernel(const double* __restrict__ vel, double* __restrict__ dirs,
                                   uint64_t n) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const double v[4] = {vel[4 * i], vel[4 * i + 1], vel[4 * i + 2], vel[4 * i + 3]};
    gg::spatial_dir(v, dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2]);
  }
}

// 12 doubles in per point (M, a, r, theta, w[4], kb[4]); 7 out (kb . da/dr,
// da/dtheta, da/dw[4], da/da).
__global__ void kerr_vjp_kernel(const double* __restrict__ in, double* __restrict__ out,
                                uint64_t n, int form) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const double* q = in + 12 * i;
    const double w[4] = {q[4], q[5], q[6], q[7]};
    const double kb[4] = {q[8], q[9], q[10], q[11]};
    double Xr = 0.0, Xth = 0.0, W[4] = {0.0, 0.0, 0.0, 0.0}, ga = 0.0;
    if (form == 0)
      gg::kerr_rhs_vjp_hand(q[0], q[1], q[2], q[3], w, kb, &Xr, &Xth, W, &ga);
    else
      gg::kerr_rhs_vjp_dual(q[0], q[1], q[2], q[3], w, kb, &Xr, &Xth, W, &ga);
    double* o = out + 7 * i;
    o[0] = Xr;
    o[1] = Xth;
    o[2] = W[0];
    o[3] = W[1];
    o[4] = W[2];
    o[5] = W[3];
    o[6] = ga;
  }
}

__global__ void step_factor_kernel(const double* __restrict__ s2, double* __restrict__ out,
                                   uint64_t n) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = gg::root10_8_over(s2[i]);
}

int launch_status() {
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? GG_OK : GG_ERR_CUDA;
}

}  // namespace

extern "C" GG_API int gg_check_procedural_sky(const double* dirs_dev, double* rgb_dev, uint64_t n,
                                              void* stream) {
  if (n == 0) return GG_OK;
  if (!dirs_dev || !rgb_dev) return GG_ERR_INVALID_ARG;
  const uint64_t blocks = (n + 255) / 256;
  sky_dir_kernel<<<(unsigned)(blocks < 4096 ? blocks : 4096), 256, 0,
                   static_cast<cudaStream_t>(stream)>>>(dirs_dev, rgb_dev, n);
  return launch_status();
}

extern "C" GG_API int gg_check_spatial_dir(const double* vel_dev, double* dirs_dev, uint64_t n,
                                           void* stream) {
  if (n == 0) return GG_OK;
  if (!vel_dev || !dirs_dev) return GG_ERR_INVALID_ARG;
  const uint64_t blocks = (n + 255) / 256;
  spatial_dir_kernel<<<(unsigned)(blocks < 4096 ? blocks : 4096), 256, 0,
                       static_cast<cudaStream_t>(stream)>>>(vel_dev, dirs_dev, n);
  return launch_status();
}

extern "C" GG_API int gg_check_kerr_vjp(const double* in_dev, double* out_dev, uint64_t n,
                                        int form, void* stream) {
  if (n == 0) return GG_OK;
  if (!in_dev || !out_dev || (form != 0 && form != 1)) return GG_ERR_INVALID_ARG;
  const uint64_t blocks = (n + 127) / 128;
  kerr_vjp_kernel<<<(unsigned)(blocks < 4096 ? blocks : 4096), 128, 0,
                    static_cast<cudaStream_t>(stream)>>>(in_dev, out_dev, n, form);
  return launch_status();
}

extern "C" GG_API int gg_check_step_factor(const double* s2_dev, double* out_dev, uint64_t n,
                                           void* stream) {
  if (n == 0) return GG_OK;
  if (!s2_dev || !out_dev) return GG_ERR_INVALID_ARG;
  const uint64_t blocks = (n + 255) / 256;
  step_factor_kernel<<<(unsigned)(blocks < 4096 ? blocks : 4096), 256, 0,
                       static_cast<cudaStream_t>(stream)>>>(s2_dev, out_dev, n);
  return launch_status();
}
