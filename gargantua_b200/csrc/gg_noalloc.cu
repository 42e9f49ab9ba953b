// gg_noalloc.cu -- a render entry point that allocates no memory.
//
// Some callers cannot let a library allocate device memory: applications
// that own all device memory through their own fixed arena or pool
// allocator, real-time or embedded hosts that forbid allocation after
// start-up, and code that must not trigger the device-wide synchronisation a
// cudaMalloc / cudaFree can cause.  gg_render_device needs a gg_ctx, and
// creating or growing one allocates (counters, a stream, events, the
// supersampling buffer).
//
// gg_render_device_noalloc takes no context.  Its scratch -- the work-queue
// and statistics counters and, for supersampled images, one linear colour
// per sample -- lives in one fixed-size file-scope device array that the CUDA
// runtime creates on each device when this library's module is loaded there
// and keeps until the process exits.  The caller passes the outputs (device
// pointers) and the stream; the kernels are the same ones gg_render_device
// launches.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>

#include "../../include/gargantua_gpu.h"
#include "gg_host.h"
#include "gg_launch.h"
#include "gg_params.h"

namespace {

constexpr size_t kScratchBytes = size_t(16) << 20;  // 16 MiB on every device
constexpr size_t kControlBytes = 256;               // DevControl, padded
static_assert(sizeof(gg::DevControl) <= kControlBytes, "control block outgrew its slot");
// supersampled renders keep 3 doubles per sample in the rest of the array
constexpr uint64_t kMaxSupersampled = (kScratchBytes - kControlBytes) / (3 * sizeof(double));

__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Device address of g_noalloc_scratch in the current device's context.  In
// host code the symbol is only a host-side handle.  The address is looked up
// on every call, with the device current, and not cached: after a
// cudaDeviceReset the module is reloaded and the array may move, and another
// context on the same device holds its own copy of the array.  Once the
// module is loaded in a context the lookup allocates nothing; the first call
// on a device loads it there.
int scratch_address(void** out) {
  void* p = nullptr;
  if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
    cudaGetLastError();
    return GG_ERR_CUDA;
  }
  *out = p;
  return GG_OK;
}

// A failed runtime call's error code stays as the thread's last error, where
// a later successful call (which checks cudaGetLastError after its launches)
// would find it: clear it before reporting the failure.
int cuda_failed() {
  cudaGetLastError();
  return GG_ERR_CUDA;
}

}  // namespace

extern "C" GG_API int gg_render_device_noalloc(const gg_metric_t* metric,
                                               const gg_camera_t* camera,
                                               const gg_disk_t* disk,
                                               const gg_integrator_t* integ,
                                               const gg_render_opts_t* opts, uint32_t width,
                                               uint32_t height, uint8_t* rgb_dev,
                                               const gg_ray_out_t* rays_dev, void* stream) {
  const int v = gg::validate_render(metric, camera, disk, integ, opts, width, height);
  if (v != GG_OK) return v;
  if (integ->precision != GG_PREC_FP64 || opts->attempt_budget != 0 ||
      opts->sky == GG_SKY_HDRI || opts->scene)  // the map and scene belong to a context
    return GG_ERR_UNSUPPORTED;
  gg::DevParams P;
  gg::make_params(metric, camera, disk, integ, opts, width, height, &P);
  const bool want_image = rgb_dev != nullptr;
  const bool need_samples = want_image && P.spp > 1;
  if (need_samples && P.n_rays > kMaxSupersampled) return GG_ERR_TOO_LARGE;

  int device = -1;
  if (cudaGetDevice(&device) != cudaSuccess) {
    cudaGetLastError();
    return GG_ERR_NO_DEVICE;
  }
  int major = 0, sms = 0;
  if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
    return cuda_failed();
  if (major != 10) return GG_ERR_NO_DEVICE;
  void* base = nullptr;
  const int st = scratch_address(&base);
  if (st != GG_OK) return st;

  gg::DevControl* ctl = static_cast<gg::DevControl*>(base);
  gg::DevOutputs O;
  std::memset(&O, 0, sizeof(O));
  if (rays_dev) {
    O.cls = rays_dev->cls;
    O.x = rays_dev->x;
    O.v = rays_dev->v;
    O.lam = rays_dev->lambda;
    O.attempts = rays_dev->attempts;
    O.accepted = rays_dev->accepted;
    O.intensity = rays_dev->intensity;
    O.color_temp = rays_dev->color_temp;
    O.rgb = rays_dev->rgb;
    O.cross = rays_dev->cross;
  }
  O.rgb8 = rgb_dev;
  O.sample_rgb = need_samples ? reinterpret_cast<double*>(static_cast<char*>(base) + kControlBytes)
                              : nullptr;

  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // the counters keep the previous call's totals: the work queue must start at 0
  if (cudaMemsetAsync(ctl, 0, sizeof(gg::DevControl), s) != cudaSuccess) return cuda_failed();
  int bps = 0;
  if (gg::trace_occupancy(P, &bps) != cudaSuccess || bps < 1) return cuda_failed();
  uint64_t grid = (uint64_t)sms * (uint64_t)bps;
  const uint64_t need_blocks = (P.n_rays + gg::kTraceBlock - 1) / gg::kTraceBlock;
  if (grid > need_blocks) grid = need_blocks;
  if (grid < 1) grid = 1;
  if (gg::launch_trace(P, O, ctl, (int)grid, s) != cudaSuccess) return cuda_failed();
  if (need_samples && gg::launch_reduce(P, O.sample_rgb, rgb_dev, sms, s) != cudaSuccess)
    return cuda_failed();
  return GG_OK;
}
