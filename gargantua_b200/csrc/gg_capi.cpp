// gg_capi.cpp -- the C ABI of libgargantua_gpu.so (include/gargantua_gpu.h).
//
// Host side of a render: validate the public POD structs, evaluate the
// per-render constants in the reference's operation order (camera frame,
// metric at the camera, horizon), manage the context's device scratch, and
// enqueue the trace kernels on the context's stream.  No function here
// aborts, throws across the ABI or falls back to the CPU.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "../../include/gargantua_gpu.h"
#include "gg_host.h"
#include "gg_launch.h"
#include "gg_params.h"
#include "gg_scene_host.h"

using gg::DevControl;
using gg::DevOutputs;
using gg::DevParams;

struct gg_ctx {
  int device = 0;
  int sms = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev_start = nullptr, ev_stop = nullptr, ev_done = nullptr;
  DevControl* ctl = nullptr;       // device counters
  DevControl* ctl_host = nullptr;  // pinned mirror
  void* samples = nullptr;         // per-sample linear colours (supersampling)
  size_t samples_cap = 0;
  void* staging = nullptr;         // device outputs of the host-buffer entry point
  size_t staging_cap = 0;
  void* queue = nullptr;           // mixed form: rays handed to the FP64 pass
  size_t queue_cap = 0;
  void* ret = nullptr;             // mixed form: rays the FP64 pass hands back
  size_t ret_cap = 0;
  // batched renders: scene table (device and pinned host mirror), kernel
  // variant, and the cached graph of the last batch shape
  void* batch_dev = nullptr;
  size_t batch_dev_cap = 0;
  void* batch_host = nullptr;
  size_t batch_host_cap = 0;
  int batch_variant = 0;
  struct BatchKey {
    uint32_t n = 0;
    uint64_t total = 0;
    int variant = -1;
    const void* queue = nullptr;
    const void* ret = nullptr;
    const void* table = nullptr;
    gg_integrator_t integ{};
    gg_render_opts_t opts{};
    int metric = -1, disk = -1;
  } batch_key;
  cudaGraphExec_t batch_exec = nullptr;
  // differentiable render: the last forward's parameters and per-ray records
  DevParams diff_P{};
  bool diff_ready = false;
  uint32_t diff_ckpt_per_ray = 0;
  void* diff_rays = nullptr;
  size_t diff_rays_cap = 0;
  void* diff_ckpt = nullptr;
  size_t diff_ckpt_cap = 0;
  void* diff_list = nullptr;  // the backward pass's sorted work list
  size_t diff_list_cap = 0;
  double* diff_grad = nullptr;       // 5 doubles, device
  double* diff_grad_host = nullptr;  // pinned
  // equirectangular sky map (gg_set_hdri), RGB float texels on the device
  float* hdri = nullptr;
  size_t hdri_cap = 0;
  uint32_t hdri_w = 0, hdri_h = 0;
  float hdri_intensity = 1.f;
  // scene of objects (gg_set_scene): primitives and hierarchy on the device
  void* scene_prims = nullptr;
  size_t scene_prims_cap = 0;
  void* scene_nodes = nullptr;
  size_t scene_nodes_cap = 0;
  bool scene_set = false;
  bool pending = false;            // stats of the last device-pointer render not read yet
  gg_stats_t last{};
  std::mutex mu;
};

// Half-width (rad) of the polar caps whose attempts the mixed form runs in
// FP64 (tuning builds override it).  Measured (mixed against FP64 DP45): the
// stress frame at 2048^2 x 4 spp takes 84.3 / 82.1 / 81.3 ms at 0.1 / 0.05 /
// 0.02 rad, and a Kerr a = 0.95 view from 10 deg off the axis spends 28 / 16 /
// 9 % of its attempts in FP64 with about the same crossing errors; but on the
// 1080p Kerr frame 0.05 rad takes the rays beyond 1e-6 from 823 to 1,056, 239
// of them not explained by the FP64 kernel's own amplification.  So 0.1.
#ifndef GG_POLE_BAND
#define GG_POLE_BAND 0.1f
#endif
// Width (M) of the radial FP64 band outside the prograde photon orbit or the
// horizon's test radius.  Measured on the 1080p Kerr frame at 0.25 / 0.35 /
// 0.5 / 0.75 M: 25.8 / 25.7 / 25.7 / 25.7 ms, and 820 / 821 / 823 / 822 rays
// beyond 1e-6, all explained by the FP64 kernel's own amplification: the band
// pass is set by its longest chains, which orbit inside any of these widths.
#ifndef GG_BAND_MARGIN
#define GG_BAND_MARGIN 0.5
#endif

namespace {

constexpr double kPi = 3.14159265358979323846;
// Renders of at least this many samples run the mixed form's hand-back
// rounds.  Measured: the 1080p Kerr view cropped to 256^2 .. 768^2 gains
// 0.6 ms with rounds, the batch benchmark's close-camera scenes (12 % of
// rays in the band) lose 1-2 ms each at every size.
#ifndef GG_HAND_BACK_MIN_RAYS
#define GG_HAND_BACK_MIN_RAYS (1ull << 20)
#endif
constexpr uint64_t kHandBackMinRays = GG_HAND_BACK_MIN_RAYS;

// ---- reference-order host math (no contraction: built -ffp-contract=off) --
struct V3 {
  double x, y, z;
};
double dot3(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
V3 normalize3(V3 v) {
  const double n = std::sqrt(dot3(v, v));
  return {v.x / n, v.y / n, v.z / n};
}
V3 cross3(V3 a, V3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

struct G5 {
  double tt, rr, thth, phph, tph;
};

// Schwarzschild::metric_tensor (schwarzschild.rs:26-43) and
// Kerr::metric_tensor (kerr.rs:61-94), evaluated at the camera.
G5 metric_at(const gg_metric_t& m, const double pos[4]) {
  G5 g{};
  double r = std::fmax(pos[1], 1e-10);
  const double theta = pos[2];
  if (m.kind == GG_METRIC_KERR) {
    const double M = m.mass, a = m.spin, a2 = a * a;
    const double ct = std::cos(theta);
    const double sigma = r * r + a * a * ct * ct;
    const double delta = r * r - 2.0 * M * r + a * a;
    const double st = std::sin(theta);
    const double sin2 = st * st;
    g.tt = -(1.0 - 2.0 * M * r / sigma);
    g.rr = sigma / delta;
    g.thth = sigma;
    g.phph = (r * r + a2 + 2.0 * M * a2 * r * sin2 / sigma) * sin2;
    g.tph = -2.0 * M * a * r * sin2 / sigma;
  } else {
    const double rs = 2.0 * m.mass;
    const double f = 1.0 - rs / r;
    const double st = std::sin(theta);
    g.tt = -f;
    g.rr = 1.0 / f;
    g.thth = r * r;
    g.phph = r * r * st * st;
    g.tph = 0.0;
  }
  return g;
}

bool finite_all(const double* p, int n) {
  for (int i = 0; i < n; ++i)
    if (!std::isfinite(p[i])) return false;
  return true;
}

// Image rows a render traces: row_offset, row_offset + row_step, ...
uint32_t rows_of(const gg_render_opts_t& o, uint32_t height) {
  const uint32_t step = o.row_step > 1 ? o.row_step : 1;
  return o.row_offset >= height ? 0u : (height - o.row_offset + step - 1) / step;
}

uint32_t spp_of(const gg_render_opts_t& o) {
  if (o.jitter_spp > 0) return o.jitter_spp;
  const uint32_t spa = o.samples_per_axis < 1 ? 1 : o.samples_per_axis;
  return spa * spa;
}

int validate(const gg_metric_t* metric, const gg_camera_t* camera, const gg_disk_t* disk,
             const gg_integrator_t* integ, const gg_render_opts_t* opts, uint32_t width,
             uint32_t height) {
  if (!metric || !camera || !integ || !opts) return GG_ERR_INVALID_ARG;
  if (metric->kind != GG_METRIC_SCHWARZSCHILD && metric->kind != GG_METRIC_KERR)
    return GG_ERR_INVALID_ARG;
  if (!(std::isfinite(metric->mass) && metric->mass > 0.0)) return GG_ERR_INVALID_ARG;
  if (metric->kind == GG_METRIC_KERR &&
      !(std::isfinite(metric->spin) && std::fabs(metric->spin) <= metric->mass))
    return GG_ERR_INVALID_ARG;
  if (!finite_all(camera->position, 4) || !finite_all(camera->look_at, 3) ||
      !finite_all(camera->up, 3))
    return GG_ERR_INVALID_ARG;
  if (!(camera->aspect > 0.0 && std::isfinite(camera->aspect))) return GG_ERR_INVALID_ARG;
  if (!(camera->fov_y_radians > 0.0 && camera->fov_y_radians < kPi)) return GG_ERR_INVALID_ARG;
  if (!(camera->position[1] > 0.0)) return GG_ERR_INVALID_ARG;
  const V3 la{camera->look_at[0], camera->look_at[1], camera->look_at[2]};
  const V3 up{camera->up[0], camera->up[1], camera->up[2]};
  if (!(dot3(la, la) > 0.0)) return GG_ERR_INVALID_ARG;
  const V3 cr = cross3(la, up);
  if (!(dot3(cr, cr) > 0.0)) return GG_ERR_INVALID_ARG;  // up parallel to look_at
  if (disk && disk->kind != GG_DISK_NONE) {
    if (disk->kind != GG_DISK_VOLUMETRIC && disk->kind != GG_DISK_THIN) return GG_ERR_INVALID_ARG;
    if (!(disk->r_inner > 0.0 && disk->r_outer >= disk->r_inner && std::isfinite(disk->r_outer)))
      return GG_ERR_INVALID_ARG;
    if (disk->kind == GG_DISK_VOLUMETRIC &&
        !(disk->scale_height > 0.0 && std::isfinite(disk->scale_height) &&
          std::isfinite(disk->density_0) && std::isfinite(disk->temperature_0)))
      return GG_ERR_INVALID_ARG;
    if (disk->kind == GG_DISK_THIN && !std::isfinite(disk->emissivity_index))
      return GG_ERR_INVALID_ARG;
  }
  if (!(integ->initial_step > 0.0 && std::isfinite(integ->initial_step))) return GG_ERR_INVALID_ARG;
  if (!(integ->min_step > 0.0 && integ->max_step >= integ->min_step &&
        std::isfinite(integ->max_step)))
    return GG_ERR_INVALID_ARG;
  if (!(integ->rtol >= 0.0 && integ->atol >= 0.0 && std::isfinite(integ->rtol) &&
        std::isfinite(integ->atol)))
    return GG_ERR_INVALID_ARG;
  if (integ->rtol > 0.0) {
    if (!(integ->atol > 0.0)) return GG_ERR_INVALID_ARG;
  } else if (!(integ->tolerance > 0.0 && std::isfinite(integ->tolerance))) {
    return GG_ERR_INVALID_ARG;
  }
  if (!(integ->max_radius > 0.0 && std::isfinite(integ->max_radius))) return GG_ERR_INVALID_ARG;
  if (!std::isfinite(integ->horizon_buffer)) return GG_ERR_INVALID_ARG;
  if (integ->max_steps < 1) return GG_ERR_INVALID_ARG;
  if (integ->precision != GG_PREC_FP64 && integ->precision != GG_PREC_MIXED)
    return GG_ERR_INVALID_ARG;
  if (integ->stepper != GG_STEPPER_REFERENCE && integ->stepper != GG_STEPPER_DP45)
    return GG_ERR_INVALID_ARG;
  if (opts->sky != GG_SKY_PROCEDURAL && opts->sky != GG_SKY_CHECKER && opts->sky != GG_SKY_HDRI)
    return GG_ERR_INVALID_ARG;
  if (opts->sky == GG_SKY_CHECKER && (opts->sky_rows < 1 || opts->sky_cols < 1))
    return GG_ERR_INVALID_ARG;
  if (opts->scene > 1) return GG_ERR_INVALID_ARG;
  if (width < 1 || height < 1) return GG_ERR_INVALID_ARG;
  const uint64_t spa = opts->samples_per_axis < 1 ? 1 : opts->samples_per_axis;
  if (opts->jitter_spp == 0 && (spa * width > 0xffffffffull || spa * height > 0xffffffffull))
    return GG_ERR_INVALID_ARG;
  const uint32_t step = opts->row_step > 1 ? opts->row_step : 1;
  if (opts->row_offset >= step || opts->row_offset >= height) return GG_ERR_INVALID_ARG;
  const uint64_t n = (uint64_t)width * rows_of(*opts, height) * spp_of(*opts);
  if (n == 0 || n > (1ull << 40)) return GG_ERR_INVALID_ARG;
  return GG_OK;
}

// Combinations the kernels implement beyond validate()'s field checks: the
// mixed form runs the full Dormand-Prince stepper (the reference's step moves
// positions by h*v_before, a first-order update whose endpoints follow the
// exact step sequence, so FP32 rounding would show at 1e-4) with a thin disk
// or none.
int supported(const gg_disk_t* disk, const gg_integrator_t* integ,
              const gg_render_opts_t* opts) {
  // scene chords: the FP64 kernels, with no disk or the volumetric one (the
  // reference's render_with_scene / render_with_disk_and_scene)
  if (opts->scene &&
      (integ->precision != GG_PREC_FP64 || (disk && disk->kind == GG_DISK_THIN)))
    return GG_ERR_UNSUPPORTED;
  if (integ->precision == GG_PREC_MIXED) {
    if (integ->stepper != GG_STEPPER_DP45) return GG_ERR_UNSUPPORTED;
    if (disk && disk->kind == GG_DISK_VOLUMETRIC) return GG_ERR_UNSUPPORTED;
  }
  return GG_OK;
}

double photon_orbit(double mass, double spin) {
  return 2.0 * mass * (1.0 + std::cos((2.0 / 3.0) * std::acos(-spin / mass)));
}

void build_params(const gg_metric_t* metric, const gg_camera_t* camera, const gg_disk_t* disk,
                  const gg_integrator_t* integ, const gg_render_opts_t* opts, uint32_t width,
                  uint32_t height, DevParams* out) {
  DevParams P;
  std::memset(&P, 0, sizeof(P));
  P.metric = metric->kind == GG_METRIC_KERR ? gg::kMetricKerr : gg::kMetricSchwarzschild;
  P.mass = metric->mass;
  P.spin = metric->kind == GG_METRIC_KERR ? metric->spin : 0.0;
  P.rs = 2.0 * metric->mass;
  if (P.metric == gg::kMetricKerr) {  // kerr.rs:427-436
    const double disc = P.mass * P.mass - P.spin * P.spin;
    P.has_horizon = disc < 0.0 ? 0 : 1;
    P.rh = disc < 0.0 ? 0.0 : P.mass + std::sqrt(disc);
    P.r_photon = photon_orbit(P.mass, P.spin);
  } else {
    P.has_horizon = 1;
    P.rh = P.rs;
    P.r_photon = 3.0 * P.mass;
  }
  P.rh_plus_buffer = P.rh + integ->horizon_buffer;
  P.initial_step = integ->initial_step;
  P.min_step = integ->min_step;
  P.max_step = integ->max_step;
  P.tolerance = integ->tolerance;
  P.max_radius = integ->max_radius;
  P.rtol = integ->rtol;
  P.atol = integ->atol;
  P.max_steps = integ->max_steps;
  P.precision = integ->precision;
  P.stepper = integ->stepper == GG_STEPPER_DP45 ? gg::kStepperDP45 : gg::kStepperReference;
  P.mass_f = (float)P.mass;
  P.spin_f = (float)P.spin;
  P.rs_f = (float)P.rs;
  P.atol_f = std::fmax((float)P.atol, 1.17549435e-38f);  // keep the scale of a 0 component > 0
  P.rtol_f = (float)P.rtol;
  {
    const double m = P.mass, a = P.spin;
    P.a2_f = (float)(a * a);
    P.m2_f = (float)(2.0 * m);
    P.mm2a2_f = (float)(-2.0 * a * a);
    P.m2a_f = (float)(2.0 * m * a);
    P.m4a_f = (float)(4.0 * m * a);
    P.m2a2_f = (float)(2.0 * m * a * a);
    P.m4a2_f = (float)(4.0 * m * a * a);
  }
  P.max_radius_hi = (float)P.max_radius;
  P.max_radius_lo = (float)(P.max_radius - (double)P.max_radius_hi);
  // FP64 band: within GG_BAND_MARGIN (0.5) M of the prograde photon orbit or
  // of the horizon test radius (the photon orbit lies outside the horizon),
  // and GG_POLE_BAND of the poles
  P.band_r = (float)(std::fmax(P.r_photon, P.rh_plus_buffer) + GG_BAND_MARGIN);
  P.pole_band = GG_POLE_BAND;

  P.width = width;
  P.height = height;
  P.jitter_spp = opts->jitter_spp;
  P.spa = opts->jitter_spp > 0 ? 1 : (opts->samples_per_axis < 1 ? 1 : opts->samples_per_axis);
  P.spp = spp_of(*opts);
  P.sub_w = width * P.spa;
  P.sub_h = height * P.spa;
  P.seed = opts->seed;
  P.row_step = opts->row_step > 1 ? opts->row_step : 1;
  P.row0 = opts->row_offset;
  P.rows = rows_of(*opts, height);
  P.n_rays = (uint64_t)width * P.rows * P.spp;
  P.inv_spp = 1.0 / (double)P.spp;

  // Camera::pixel_direction frame (camera.rs:20-29)
  const V3 la{camera->look_at[0], camera->look_at[1], camera->look_at[2]};
  const V3 upv{camera->up[0], camera->up[1], camera->up[2]};
  const V3 forward = normalize3(la);
  const V3 right = normalize3(cross3(forward, upv));
  const V3 up2 = normalize3(cross3(right, forward));
  P.cam_forward[0] = forward.x; P.cam_forward[1] = forward.y; P.cam_forward[2] = forward.z;
  P.cam_right[0] = right.x; P.cam_right[1] = right.y; P.cam_right[2] = right.z;
  P.cam_up[0] = up2.x; P.cam_up[1] = up2.y; P.cam_up[2] = up2.z;
  P.half_h = std::tan(camera->fov_y_radians / 2.0);
  P.half_w = P.half_h * camera->aspect;
  // local spherical frame and metric at the camera (ray.rs:29-48)
  for (int i = 0; i < 4; ++i) P.cam_pos[i] = camera->position[i];
  const double theta = camera->position[2], phi = camera->position[3];
  const double st = std::sin(theta), ct = std::cos(theta);
  const double sp = std::sin(phi), cp = std::cos(phi);
  P.r_hat[0] = st * cp; P.r_hat[1] = st * sp; P.r_hat[2] = ct;
  P.theta_hat[0] = ct * cp; P.theta_hat[1] = ct * sp; P.theta_hat[2] = -st;
  P.phi_hat[0] = -sp; P.phi_hat[1] = cp; P.phi_hat[2] = 0.0;
  const G5 g = metric_at(*metric, camera->position);
  P.cam_g_tt = g.tt;
  P.cam_g_rr = g.rr;
  P.cam_g_thth = g.thth;
  P.cam_g_phph = g.phph;
  P.sqrt_g_rr = std::sqrt(g.rr);
  P.sqrt_g_thth = std::sqrt(g.thth);
  P.sqrt_g_phph = std::sqrt(g.phph);
  P.sqrt_neg_gtt_obs = std::sqrt(std::fmax(-g.tt, 0.0));  // tracer.rs:93-94

  P.disk = disk ? disk->kind : GG_DISK_NONE;
  if (disk) {
    P.r_inner = disk->r_inner;
    P.r_outer = disk->r_outer;
    P.scale_height = disk->scale_height;
    P.density_0 = disk->density_0;
    P.temperature_0 = disk->temperature_0;
    P.emissivity_index = disk->emissivity_index;
  }
  P.sky = opts->sky;
  P.sky_rows = opts->sky_rows;
  P.sky_cols = opts->sky_cols;
  P.sky_seed = opts->sky_seed;
  P.cell_h = kPi / (double)(opts->sky_rows ? opts->sky_rows : 1);
  P.cell_w = (2.0 * kPi) / (double)(opts->sky_cols ? opts->sky_cols : 1);
  P.attempt_budget = opts->attempt_budget;
  P.scene = opts->scene;
  *out = P;
}

// The context's sky map into P for GG_SKY_HDRI renders; no map set is an
// invalid argument.
int attach_sky_map(const gg_ctx* c, DevParams* P) {
  if (P->scene) {  // the context's scene, likewise
    if (!c->scene_set) return GG_ERR_INVALID_ARG;
    P->prims = static_cast<const gg::ScenePrim*>(c->scene_prims);
    P->nodes = static_cast<const gg::SceneNode*>(c->scene_nodes);
  }
  if (P->sky != gg::kSkyHdri) return GG_OK;
  if (!c->hdri) return GG_ERR_INVALID_ARG;
  P->hdri = c->hdri;
  P->hdri_w = c->hdri_w;
  P->hdri_h = c->hdri_h;
  P->hdri_intensity = c->hdri_intensity;
  return GG_OK;
}

int grow_pinned(void** buf, size_t* cap, size_t need) {
  if (need <= *cap) return GG_OK;
  if (*buf) cudaFreeHost(*buf);
  *buf = nullptr;
  *cap = 0;
  const size_t want = need + need / 4;
  if (cudaMallocHost(buf, want) != cudaSuccess) {
    cudaGetLastError();
    *buf = nullptr;
    return GG_ERR_OOM;
  }
  *cap = want;
  return GG_OK;
}

int grow(void** buf, size_t* cap, size_t need) {
  if (need <= *cap) return GG_OK;
  if (*buf) cudaFree(*buf);
  *buf = nullptr;
  *cap = 0;
  size_t want = need + need / 4;
  if (cudaMalloc(buf, want) != cudaSuccess) {
    cudaGetLastError();
    if (cudaMalloc(buf, need) != cudaSuccess) {
      cudaGetLastError();
      *buf = nullptr;
      return GG_ERR_OOM;
    }
    want = need;
  }
  *cap = want;
  return GG_OK;
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Enqueues one render with device outputs O on `stream`.
int enqueue(gg_ctx* ctx, const DevParams& P, DevOutputs O, bool want_image,
            cudaStream_t stream) {
  if (cudaStreamWaitEvent(stream, ctx->ev_done, 0) != cudaSuccess) return GG_ERR_CUDA;
  if (want_image && P.spp > 1) {
    const int st = grow(&ctx->samples, &ctx->samples_cap, sizeof(double) * 3 * P.n_rays);
    if (st != GG_OK) return st;
    O.sample_rgb = static_cast<double*>(ctx->samples);
  } else {
    O.sample_rgb = nullptr;
  }
  if (!want_image) O.rgb8 = nullptr;
  const bool mixed = P.precision == GG_PREC_MIXED;
  O.queue = nullptr;
  O.queue_cap = 0;
  O.ret = nullptr;
  O.ret_cap = 0;
  // The hand-back to the FP32 stepper (two more launches) runs in renders of
  // at least kHandBackMinRays samples without an attempt budget (whose
  // bookkeeping stays in the single round).  Measured: a 1080p frame gains
  // (29.9 -> 29.5 ms), while renders of 64^2..512^2 lose about 1 ms each to
  // the extra launches' tails.
  const bool rounds = mixed && P.attempt_budget == 0 && P.n_rays >= kHandBackMinRays;
  if (mixed) {  // every ray can be handed over (and back) at most once per round
    int st = grow(&ctx->queue, &ctx->queue_cap, sizeof(gg::QueuedRay) * P.n_rays);
    if (st != GG_OK) return st;
    O.queue = static_cast<gg::QueuedRay*>(ctx->queue);
    O.queue_cap = P.n_rays;
    if (rounds) {
      st = grow(&ctx->ret, &ctx->ret_cap, sizeof(gg::QueuedRay) * P.n_rays);
      if (st != GG_OK) return st;
      O.ret = static_cast<gg::QueuedRay*>(ctx->ret);
      O.ret_cap = P.n_rays;
    }
  }
  if (cudaMemsetAsync(ctx->ctl, 0, sizeof(DevControl), stream) != cudaSuccess) return GG_ERR_CUDA;
  int bps = 0;
  const cudaError_t oe = mixed ? gg::mixed_occupancy(P, &bps) : gg::trace_occupancy(P, &bps);
  if (oe != cudaSuccess || bps < 1) return GG_ERR_CUDA;
  uint64_t grid = (uint64_t)ctx->sms * (uint64_t)bps;
  const uint64_t need_blocks = (P.n_rays + gg::kTraceBlock - 1) / gg::kTraceBlock;
  if (grid > need_blocks) grid = need_blocks;
  if (grid < 1) grid = 1;
  int qbps = 0, rbps = 0;
  if (mixed && (gg::queue_trace_occupancy(P, &qbps) != cudaSuccess || qbps < 1))
    return GG_ERR_CUDA;
  if (rounds && (gg::mixed_occupancy(P, &rbps, nullptr, 0, true) != cudaSuccess || rbps < 1))
    return GG_ERR_CUDA;
  if (cudaEventRecord(ctx->ev_start, stream) != cudaSuccess) return GG_ERR_CUDA;
  if (mixed) {
    if (gg::launch_mixed(P, O, ctx->ctl, (int)grid, stream) != cudaSuccess) return GG_ERR_CUDA;
    // the queues' lengths are only known on the device: full persistent
    // grids, whose surplus warps find the queue empty and exit
    DevParams P1 = P;
    P1.hand_back = rounds ? 1u : 0u;
    if (gg::launch_queue_trace(P1, O, ctx->ctl, ctx->sms * qbps, stream) != cudaSuccess)
      return GG_ERR_CUDA;
    if (rounds) {
      if (gg::launch_next_round(ctx->ctl, stream) != cudaSuccess ||
          gg::launch_mixed(P, O, ctx->ctl, ctx->sms * rbps, stream, nullptr, 0, true) !=
              cudaSuccess ||
          gg::launch_queue_trace(P, O, ctx->ctl, ctx->sms * qbps, stream) != cudaSuccess)
        return GG_ERR_CUDA;
    }
  } else if (gg::launch_trace(P, O, ctx->ctl, (int)grid, stream) != cudaSuccess) {
    return GG_ERR_CUDA;
  }
  if (cudaEventRecord(ctx->ev_stop, stream) != cudaSuccess) return GG_ERR_CUDA;
  if (O.sample_rgb && O.rgb8) {
    if (gg::launch_reduce(P, O.sample_rgb, O.rgb8, ctx->sms, stream) != cudaSuccess)
      return GG_ERR_CUDA;
  }
  if (cudaMemcpyAsync(ctx->ctl_host, ctx->ctl, sizeof(DevControl), cudaMemcpyDeviceToHost,
                      stream) != cudaSuccess)
    return GG_ERR_CUDA;
  if (cudaEventRecord(ctx->ev_done, stream) != cudaSuccess) return GG_ERR_CUDA;
  ctx->pending = true;
  return GG_OK;
}

// Waits for the last render and folds its counters into ctx->last.
int collect(gg_ctx* ctx) {
  if (!ctx->pending) return GG_OK;
  if (cudaEventSynchronize(ctx->ev_done) != cudaSuccess) return GG_ERR_CUDA;
  ctx->pending = false;
  const DevControl& c = *ctx->ctl_host;
  gg_stats_t s{};
  s.attempts = c.attempts;
  s.accepted = c.accepted;
  for (int k = 0; k < GG_N_CLASSES; ++k) {
    s.class_count[k] = c.class_count[k];
    s.rays += c.class_count[k];
  }
  s.fp64_rays = c.band_total + c.queued;
  s.fp64_attempts = c.fp64_attempts;
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop) == cudaSuccess) s.kernel_ms = ms;
  ctx->last = s;
  if (c.queue_overflow) return GG_ERR_OOM;
  return c.abort ? GG_ERR_BUDGET : GG_OK;
}

struct Lock {
  explicit Lock(gg_ctx* c) : g(c->mu) { cudaSetDevice(c->device); }
  std::lock_guard<std::mutex> g;
};

// ---- batched renders --------------------------------------------------------
struct BatchLaunch {
  DevParams P0;  // the batch's common parameters (integrator, sky kind), n_rays = total
  DevOutputs O0;  // the FP64 band queue
  gg::BatchTable table;
  size_t table_bytes = 0;  // bytes of the scene table + prefix array to upload
  uint64_t total = 0;
  uint64_t pixels = 0;
  int grid = 0, qgrid = 0, rgrid = 0;
  bool rounds = false;  // hand rays back from the FP64 pass (kHandBackMinRays)
};

// Validates the batch, writes the scene table (per-scene parameters and
// image pointers into rgb_dev, prefix sums of sample counts) to the pinned
// mirror, grows the device table and the band queue, and sizes the grids.
int batch_prepare(gg_ctx* c, const gg_scene_t* scenes, uint32_t n, const gg_integrator_t* integ,
                  const gg_render_opts_t* opts, uint8_t* rgb_dev, int variant, BatchLaunch* L) {
  if (!scenes || n == 0 || !integ || !opts) return GG_ERR_INVALID_ARG;
  if (integ->precision != GG_PREC_MIXED || integ->stepper != GG_STEPPER_DP45)
    return GG_ERR_UNSUPPORTED;
  if (opts->samples_per_axis > 1 || opts->jitter_spp > 0 || opts->attempt_budget != 0 ||
      opts->row_step > 1 || opts->sky == GG_SKY_HDRI || opts->scene)
    return GG_ERR_UNSUPPORTED;
  const int kind = scenes[0].metric.kind, disk_kind = scenes[0].disk.kind;
  if (disk_kind != GG_DISK_NONE && disk_kind != GG_DISK_THIN) return GG_ERR_UNSUPPORTED;
  for (uint32_t k = 0; k < n; ++k) {
    if (scenes[k].metric.kind != kind || scenes[k].disk.kind != disk_kind)
      return GG_ERR_UNSUPPORTED;
    gg_render_opts_t o = *opts;
    o.sky_seed = scenes[k].sky_seed;
    const gg_disk_t* d = disk_kind == GG_DISK_NONE ? nullptr : &scenes[k].disk;
    const int v = validate(&scenes[k].metric, &scenes[k].camera, d, integ, &o, scenes[k].width,
                           scenes[k].height);
    if (v != GG_OK) return v;
  }
  const size_t off_first = align256(sizeof(gg::BatchScene) * n);
  L->table_bytes = off_first + sizeof(uint64_t) * (n + 1);
  int st = grow_pinned(&c->batch_host, &c->batch_host_cap, L->table_bytes);
  if (st != GG_OK) return st;
  st = grow(&c->batch_dev, &c->batch_dev_cap, L->table_bytes);
  if (st != GG_OK) return st;
  auto* T = static_cast<gg::BatchScene*>(c->batch_host);
  auto* first = reinterpret_cast<uint64_t*>(static_cast<char*>(c->batch_host) + off_first);
  uint64_t total = 0, pix = 0;
  for (uint32_t k = 0; k < n; ++k) {
    gg_render_opts_t o = *opts;
    o.sky_seed = scenes[k].sky_seed;
    const gg_disk_t* d = disk_kind == GG_DISK_NONE ? nullptr : &scenes[k].disk;
    build_params(&scenes[k].metric, &scenes[k].camera, d, integ, &o, scenes[k].width,
                 scenes[k].height, &T[k].P);
    std::memset(&T[k].O, 0, sizeof(T[k].O));
    T[k].O.rgb8 = rgb_dev ? rgb_dev + 3 * pix : nullptr;
    first[k] = total;
    total += T[k].P.n_rays;
    pix += (uint64_t)scenes[k].width * scenes[k].height;
  }
  first[n] = total;
  L->total = total;
  L->pixels = pix;
  L->P0 = T[0].P;
  L->P0.n_rays = total;
  st = grow(&c->queue, &c->queue_cap, sizeof(gg::QueuedRay) * total);
  if (st != GG_OK) return st;
  L->rounds = total >= kHandBackMinRays;
  std::memset(&L->O0, 0, sizeof(L->O0));
  L->O0.queue = static_cast<gg::QueuedRay*>(c->queue);
  L->O0.queue_cap = total;
  if (L->rounds) {
    st = grow(&c->ret, &c->ret_cap, sizeof(gg::QueuedRay) * total);
    if (st != GG_OK) return st;
    L->O0.ret = static_cast<gg::QueuedRay*>(c->ret);
    L->O0.ret_cap = total;
  }
  L->table.scenes = static_cast<const gg::BatchScene*>(c->batch_dev);
  L->table.first = reinterpret_cast<const uint64_t*>(static_cast<char*>(c->batch_dev) + off_first);
  L->table.n = n;
  int bps = 0, qbps = 0;
  if (gg::mixed_occupancy(L->P0, &bps, &L->table, variant) != cudaSuccess || bps < 1)
    return GG_ERR_CUDA;
  if (gg::queue_trace_occupancy(L->P0, &qbps) != cudaSuccess || qbps < 1) return GG_ERR_CUDA;
  int rbps = 0;
  if (gg::mixed_occupancy(L->P0, &rbps, &L->table, 0, true) != cudaSuccess || rbps < 1)
    return GG_ERR_CUDA;
  L->rgrid = c->sms * rbps;
  uint64_t grid = (uint64_t)c->sms * bps;
  const uint64_t need_blocks = (total + gg::kTraceBlock - 1) / gg::kTraceBlock;
  if (grid > need_blocks) grid = need_blocks;
  L->grid = (int)(grid < 1 ? 1 : grid);
  L->qgrid = c->sms * qbps;
  return GG_OK;
}

// The batch's device work on `s`: upload the table, reset the counters, the
// mixed launch, the FP64 band pass (handing rays that leave the band back),
// the FP32 pass over those and a last FP64 pass, the counters back to the
// pinned mirror.
// Runs directly, or under stream capture to build the batch graph.
int batch_body(gg_ctx* c, const BatchLaunch& L, int variant, cudaStream_t s) {
  if (cudaMemcpyAsync(c->batch_dev, c->batch_host, L.table_bytes, cudaMemcpyHostToDevice, s) !=
      cudaSuccess)
    return GG_ERR_CUDA;
  if (cudaMemsetAsync(c->ctl, 0, sizeof(DevControl), s) != cudaSuccess) return GG_ERR_CUDA;
  if (gg::launch_mixed(L.P0, L.O0, c->ctl, L.grid, s, &L.table, variant) != cudaSuccess)
    return GG_ERR_CUDA;
  DevParams P1 = L.P0;
  P1.hand_back = L.rounds ? 1u : 0u;
  if (gg::launch_queue_trace(P1, L.O0, c->ctl, L.qgrid, s, &L.table) != cudaSuccess)
    return GG_ERR_CUDA;
  if (L.rounds &&
      (gg::launch_next_round(c->ctl, s) != cudaSuccess ||
       gg::launch_mixed(L.P0, L.O0, c->ctl, L.rgrid, s, &L.table, 0, true) != cudaSuccess ||
       gg::launch_queue_trace(L.P0, L.O0, c->ctl, L.qgrid, s, &L.table) != cudaSuccess))
    return GG_ERR_CUDA;
  if (cudaMemcpyAsync(c->ctl_host, c->ctl, sizeof(DevControl), cudaMemcpyDeviceToHost, s) !=
      cudaSuccess)
    return GG_ERR_CUDA;
  return GG_OK;
}

// One batched render into rgb_dev on `stream` through the cached graph.
int batch_render(gg_ctx* c, const gg_scene_t* scenes, uint32_t n, const gg_integrator_t* integ,
                 const gg_render_opts_t* opts, uint8_t* rgb_dev, cudaStream_t stream) {
  // the pinned table is rewritten: the previous render must have read it
  if (cudaEventSynchronize(c->ev_done) != cudaSuccess) return GG_ERR_CUDA;
  const int variant = c->batch_variant;
  BatchLaunch L;
  int st = batch_prepare(c, scenes, n, integ, opts, rgb_dev, variant, &L);
  if (st != GG_OK) return st;
  gg_ctx::BatchKey key;
  key.n = n;
  key.total = L.total;
  key.variant = variant;
  key.queue = c->queue;
  key.ret = c->ret;
  key.table = c->batch_dev;
  key.integ = *integ;
  key.opts = *opts;
  key.opts.sky_seed = 0;
  key.metric = scenes[0].metric.kind;
  key.disk = scenes[0].disk.kind;
  const bool same = c->batch_exec && key.n == c->batch_key.n &&
                    key.total == c->batch_key.total && key.variant == c->batch_key.variant &&
                    key.queue == c->batch_key.queue && key.ret == c->batch_key.ret &&
                    key.table == c->batch_key.table &&
                    key.metric == c->batch_key.metric && key.disk == c->batch_key.disk &&
                    std::memcmp(&key.integ, &c->batch_key.integ, sizeof(key.integ)) == 0 &&
                    std::memcmp(&key.opts, &c->batch_key.opts, sizeof(key.opts)) == 0;
  if (!same) {
    if (c->batch_exec) cudaGraphExecDestroy(c->batch_exec);
    c->batch_exec = nullptr;
    if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
      return GG_ERR_CUDA;
    st = batch_body(c, L, variant, c->stream);
    cudaGraph_t g = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(c->stream, &g);
    if (st != GG_OK || ce != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      return st != GG_OK ? st : GG_ERR_CUDA;
    }
    const cudaError_t ie = cudaGraphInstantiate(&c->batch_exec, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) {
      c->batch_exec = nullptr;
      return GG_ERR_CUDA;
    }
    c->batch_key = key;
  }
  if (cudaEventRecord(c->ev_start, stream) != cudaSuccess) return GG_ERR_CUDA;
  if (cudaGraphLaunch(c->batch_exec, stream) != cudaSuccess) return GG_ERR_CUDA;
  if (cudaEventRecord(c->ev_stop, stream) != cudaSuccess) return GG_ERR_CUDA;
  if (cudaEventRecord(c->ev_done, stream) != cudaSuccess) return GG_ERR_CUDA;
  c->pending = true;
  return GG_OK;
}

uint64_t batch_pixels(const gg_scene_t* scenes, uint32_t n) {
  uint64_t p = 0;
  for (uint32_t k = 0; k < n; ++k) p += (uint64_t)scenes[k].width * scenes[k].height;
  return p;
}

}  // namespace

namespace gg {

int validate_render(const gg_metric_t* metric, const gg_camera_t* camera, const gg_disk_t* disk,
                    const gg_integrator_t* integ, const gg_render_opts_t* opts, uint32_t width,
                    uint32_t height) {
  return validate(metric, camera, disk, integ, opts, width, height);
}

void make_params(const gg_metric_t* metric, const gg_camera_t* camera, const gg_disk_t* disk,
                 const gg_integrator_t* integ, const gg_render_opts_t* opts, uint32_t width,
                 uint32_t height, DevParams* out) {
  build_params(metric, camera, disk, integ, opts, width, height, out);
}

}  // namespace gg

extern "C" {

GG_API const char* gg_version(void) { return "gargantua_b200 0.1.0 (sm_100a)"; }

GG_API const char* gg_strerror(int status) {
  switch (status) {
    case GG_OK: return "ok";
    case GG_ERR_INVALID_ARG: return "invalid argument";
    case GG_ERR_CUDA: return "CUDA runtime error";
    case GG_ERR_OOM: return "device out of memory";
    case GG_ERR_BUDGET: return "attempt budget exhausted";
    case GG_ERR_UNSUPPORTED: return "unsupported combination";
    case GG_ERR_NO_DEVICE: return "no sm_100 CUDA device";
    case GG_ERR_TOO_LARGE: return "render exceeds the fixed no-allocation scratch";
    default: return "unknown status";
  }
}

GG_API int gg_struct_size(const char* name) {
  if (!name) return -1;
  struct {
    const char* n;
    int s;
  } t[] = {{"gg_metric_t", (int)sizeof(gg_metric_t)},
           {"gg_camera_t", (int)sizeof(gg_camera_t)},
           {"gg_disk_t", (int)sizeof(gg_disk_t)},
           {"gg_integrator_t", (int)sizeof(gg_integrator_t)},
           {"gg_render_opts_t", (int)sizeof(gg_render_opts_t)},
           {"gg_ray_out_t", (int)sizeof(gg_ray_out_t)},
           {"gg_stats_t", (int)sizeof(gg_stats_t)},
           {"gg_scene_t", (int)sizeof(gg_scene_t)},
           {"gg_prim_t", (int)sizeof(gg_prim_t)},
           // bytes that reach the device per render as kernel parameters
           {"launch_params", (int)(sizeof(DevParams) + sizeof(DevOutputs) + sizeof(void*))}};
  for (auto& e : t)
    if (std::strcmp(e.n, name) == 0) return e.s;
  return -1;
}

GG_API int gg_metric_schwarzschild(gg_metric_t* out, double mass) {
  if (!out) return GG_ERR_INVALID_ARG;
  std::memset(out, 0, sizeof(*out));
  out->kind = GG_METRIC_SCHWARZSCHILD;
  out->mass = mass;
  return (std::isfinite(mass) && mass > 0.0) ? GG_OK : GG_ERR_INVALID_ARG;
}

GG_API int gg_metric_kerr(gg_metric_t* out, double mass, double spin) {
  if (!out) return GG_ERR_INVALID_ARG;
  std::memset(out, 0, sizeof(*out));
  out->kind = GG_METRIC_KERR;
  out->mass = mass;
  if (!(std::isfinite(mass) && mass > 0.0)) return GG_ERR_INVALID_ARG;  // kerr.rs:30
  const double max_spin = mass * 0.9999;                                  // kerr.rs:31-32
  out->spin = spin < -max_spin ? -max_spin : (spin > max_spin ? max_spin : spin);
  return std::isfinite(spin) ? GG_OK : GG_ERR_INVALID_ARG;
}

GG_API void gg_integrator_default(gg_integrator_t* out) {
  if (!out) return;
  std::memset(out, 0, sizeof(*out));
  out->initial_step = 0.1;  // geodesic.rs:170-181
  out->min_step = 1e-8;
  out->max_step = 1.0;
  out->tolerance = 1e-6;
  out->max_radius = 200.0;  // renderer.rs:264
  out->horizon_buffer = 0.01;
  out->max_steps = 5000;    // renderer.rs:265
  out->precision = GG_PREC_FP64;
}

GG_API void gg_disk_default(gg_disk_t* out) {
  if (!out) return;
  std::memset(out, 0, sizeof(*out));
  out->kind = GG_DISK_VOLUMETRIC;  // disk.rs:21-31
  out->r_inner = 6.0;
  out->r_outer = 20.0;
  out->scale_height = 1.0;
  out->density_0 = 1.0;
  out->temperature_0 = 1.0;
  out->emissivity_index = 3.0;
}

GG_API void gg_render_opts_default(gg_render_opts_t* out) {
  if (!out) return;
  std::memset(out, 0, sizeof(*out));
  out->samples_per_axis = 1;
  out->sky = GG_SKY_PROCEDURAL;
  out->sky_rows = 18;
  out->sky_cols = 36;
}

GG_API int gg_camera_inclined(gg_camera_t* out, double r, double inclination_rad,
                              double fov_y_radians, double aspect) {
  if (!out) return GG_ERR_INVALID_ARG;
  std::memset(out, 0, sizeof(*out));
  out->position[0] = 0.0;
  out->position[1] = r;
  out->position[2] = inclination_rad;
  out->position[3] = 0.0;
  out->look_at[0] = -std::sin(inclination_rad);
  out->look_at[1] = 0.0;
  out->look_at[2] = -std::cos(inclination_rad);
  out->up[2] = 1.0;
  out->fov_y_radians = fov_y_radians;
  out->aspect = aspect;
  const bool ok = r > 0.0 && std::isfinite(r) && inclination_rad > 0.0 &&
                  inclination_rad < kPi && fov_y_radians > 0.0 && fov_y_radians < kPi &&
                  aspect > 0.0 && std::isfinite(aspect);
  return ok ? GG_OK : GG_ERR_INVALID_ARG;
}

GG_API double gg_kerr_isco(double mass, double spin) {
  // Bardeen, Press & Teukolsky (1972), prograde orbit.
  const double a = spin / mass;
  const double z1 = 1.0 + std::cbrt(1.0 - a * a) * (std::cbrt(1.0 + a) + std::cbrt(1.0 - a));
  const double z2 = std::sqrt(3.0 * a * a + z1 * z1);
  return mass * (3.0 + z2 - std::sqrt((3.0 - z1) * (3.0 + z1 + 2.0 * z2)));
}

GG_API double gg_kerr_photon_orbit(double mass, double spin) { return photon_orbit(mass, spin); }

GG_API int gg_validate(const gg_metric_t* metric, const gg_camera_t* camera,
                       const gg_disk_t* disk, const gg_integrator_t* integ,
                       const gg_render_opts_t* opts, uint32_t width, uint32_t height) {
  return validate(metric, camera, disk, integ, opts, width, height);
}

GG_API int gg_create(gg_ctx** out, int device) {
  if (!out) return GG_ERR_INVALID_ARG;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) {
    cudaGetLastError();
    return GG_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= count) return GG_ERR_INVALID_ARG;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return GG_ERR_CUDA;
  if (prop.major != 10) return GG_ERR_NO_DEVICE;  // built for sm_100a only
  if (cudaSetDevice(device) != cudaSuccess) return GG_ERR_CUDA;
  gg_ctx* c = new (std::nothrow) gg_ctx();
  if (!c) return GG_ERR_OOM;
  c->device = device;
  c->sms = prop.multiProcessorCount;
  bool ok = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreate(&c->ev_start) == cudaSuccess &&
            cudaEventCreate(&c->ev_stop) == cudaSuccess &&
            cudaEventCreateWithFlags(&c->ev_done, cudaEventDisableTiming) == cudaSuccess &&
            cudaMalloc(&c->ctl, sizeof(DevControl)) == cudaSuccess &&
            cudaMallocHost(&c->ctl_host, sizeof(DevControl)) == cudaSuccess;
  if (!ok) {
    gg_destroy(c);
    return GG_ERR_CUDA;
  }
  std::memset(c->ctl_host, 0, sizeof(DevControl));
  cudaEventRecord(c->ev_done, c->stream);
  *out = c;
  return GG_OK;
}

GG_API int gg_destroy(gg_ctx* c) {
  if (!c) return GG_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->pending && c->ev_done) cudaEventSynchronize(c->ev_done);
  if (c->samples) cudaFree(c->samples);
  if (c->staging) cudaFree(c->staging);
  if (c->queue) cudaFree(c->queue);
  if (c->ret) cudaFree(c->ret);
  if (c->batch_exec) cudaGraphExecDestroy(c->batch_exec);
  if (c->batch_dev) cudaFree(c->batch_dev);
  if (c->batch_host) cudaFreeHost(c->batch_host);
  if (c->diff_rays) cudaFree(c->diff_rays);
  if (c->diff_ckpt) cudaFree(c->diff_ckpt);
  if (c->diff_list) cudaFree(c->diff_list);
  if (c->diff_grad) cudaFree(c->diff_grad);
  if (c->diff_grad_host) cudaFreeHost(c->diff_grad_host);
  if (c->hdri) cudaFree(c->hdri);
  if (c->scene_prims) cudaFree(c->scene_prims);
  if (c->scene_nodes) cudaFree(c->scene_nodes);
  if (c->ctl) cudaFree(c->ctl);
  if (c->ctl_host) cudaFreeHost(c->ctl_host);
  if (c->ev_start) cudaEventDestroy(c->ev_start);
  if (c->ev_stop) cudaEventDestroy(c->ev_stop);
  if (c->ev_done) cudaEventDestroy(c->ev_done);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return GG_OK;
}

GG_API void* gg_stream(gg_ctx* c) { return c ? (void*)c->stream : nullptr; }

GG_API int gg_last_stats(gg_ctx* c, gg_stats_t* out) {
  if (!c || !out) return GG_ERR_INVALID_ARG;
  Lock lock(c);
  const int st = collect(c);
  *out = c->last;
  return st == GG_ERR_BUDGET ? GG_OK : st;
}

GG_API int gg_measure_fma_peak(gg_ctx* c, int fp64, double* flops) {
  if (!c || !flops) return GG_ERR_INVALID_ARG;
  Lock lock(c);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) return GG_ERR_CUDA;
  return gg::measure_fma_peak(fp64, c->sms, flops) == cudaSuccess ? GG_OK : GG_ERR_CUDA;
}

GG_API int gg_render_device(gg_ctx* c, const gg_metric_t* metric, const gg_camera_t* camera,
                            const gg_disk_t* disk, const gg_integrator_t* integ,
                            const gg_render_opts_t* opts, uint32_t width, uint32_t height,
                            uint8_t* rgb_dev, const gg_ray_out_t* rays_dev, void* stream) {
  if (!c) return GG_ERR_INVALID_ARG;
  const int v = validate(metric, camera, disk, integ, opts, width, height);
  if (v != GG_OK) return v;
  const int sup = supported(disk, integ, opts);
  if (sup != GG_OK) return sup;
  DevParams P;
  build_params(metric, camera, disk, integ, opts, width, height, &P);
  Lock lock(c);
  const int sky = attach_sky_map(c, &P);
  if (sky != GG_OK) return sky;
  DevOutputs O;
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
  // NULL is CUDA's default stream, as for any CUDA API taking a stream
  return enqueue(c, P, O, rgb_dev != nullptr, static_cast<cudaStream_t>(stream));
}

GG_API int gg_render_batch_device(gg_ctx* c, const gg_scene_t* scenes, uint32_t n,
                                  const gg_integrator_t* integ, const gg_render_opts_t* opts,
                                  uint8_t* rgb_dev, void* stream) {
  if (!c || !rgb_dev) return GG_ERR_INVALID_ARG;
  Lock lock(c);
  return batch_render(c, scenes, n, integ, opts, rgb_dev, static_cast<cudaStream_t>(stream));
}

GG_API int gg_render_batch(gg_ctx* c, const gg_scene_t* scenes, uint32_t n,
                           const gg_integrator_t* integ, const gg_render_opts_t* opts,
                           uint8_t* const* rgb_out) {
  if (!c || !scenes || n == 0 || !rgb_out) return GG_ERR_INVALID_ARG;
  for (uint32_t k = 0; k < n; ++k)
    if (!rgb_out[k]) return GG_ERR_INVALID_ARG;
  Lock lock(c);
  if (cudaEventSynchronize(c->ev_done) != cudaSuccess) return GG_ERR_CUDA;  // staging reuse
  int st = grow(&c->staging, &c->staging_cap, 3 * batch_pixels(scenes, n));
  if (st != GG_OK) return st;
  uint8_t* dev = static_cast<uint8_t*>(c->staging);
  st = batch_render(c, scenes, n, integ, opts, dev, c->stream);
  if (st != GG_OK) return st;
  uint64_t off = 0;
  for (uint32_t k = 0; k < n; ++k) {
    const size_t bytes = 3ull * scenes[k].width * scenes[k].height;
    if (cudaMemcpyAsync(rgb_out[k], dev + off, bytes, cudaMemcpyDeviceToHost, c->stream) !=
        cudaSuccess)
      return GG_ERR_CUDA;
    off += bytes;
  }
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) return GG_ERR_CUDA;
  return collect(c);
}

static_assert(GG_BATCH_VARIANTS == gg::kBatchVariants, "batch variant count");

GG_API int gg_batch_autotune(gg_ctx* c, const gg_scene_t* scenes, uint32_t n,
                             const gg_integrator_t* integ, const gg_render_opts_t* opts,
                             int* variant_out, double* ms_out) {
  if (!c || !scenes || n == 0) return GG_ERR_INVALID_ARG;
  Lock lock(c);
  if (cudaEventSynchronize(c->ev_done) != cudaSuccess) return GG_ERR_CUDA;
  int st = grow(&c->staging, &c->staging_cap, 3 * batch_pixels(scenes, n));
  if (st != GG_OK) return st;
  uint8_t* dev = static_cast<uint8_t*>(c->staging);
  int best = 0;
  double best_ms = 1e300;
  for (int v = 0; v < GG_BATCH_VARIANTS; ++v) {
    double vms = 1e300;
    for (int rep = 0; rep < 2; ++rep) {  // the first run of a variant also loads its code
      BatchLaunch L;
      st = batch_prepare(c, scenes, n, integ, opts, dev, v, &L);
      if (st != GG_OK) return st;
      if (cudaEventRecord(c->ev_start, c->stream) != cudaSuccess) return GG_ERR_CUDA;
      st = batch_body(c, L, v, c->stream);
      if (st != GG_OK) return st;
      if (cudaEventRecord(c->ev_stop, c->stream) != cudaSuccess) return GG_ERR_CUDA;
      if (cudaStreamSynchronize(c->stream) != cudaSuccess) return GG_ERR_CUDA;
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, c->ev_start, c->ev_stop) != cudaSuccess) return GG_ERR_CUDA;
      if (ms < vms) vms = ms;
    }
    if (ms_out) ms_out[v] = vms;
    if (vms < best_ms) {
      best_ms = vms;
      best = v;
    }
  }
  c->batch_variant = best;
  c->pending = false;
  cudaEventRecord(c->ev_done, c->stream);
  if (variant_out) *variant_out = best;
  return GG_OK;
}

GG_API int gg_set_hdri(gg_ctx* c, const float* rgb, uint32_t width, uint32_t height,
                       float intensity) {
  if (!c || !rgb || width < 1 || height < 1 || !std::isfinite(intensity))
    return GG_ERR_INVALID_ARG;
  const uint64_t texels = (uint64_t)width * height;
  if (texels > (1ull << 32)) return GG_ERR_INVALID_ARG;
  const size_t bytes = texels * 3 * sizeof(float);
  Lock lock(c);
  // renders in flight may read the old map
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) return GG_ERR_CUDA;
  if (cudaEventSynchronize(c->ev_done) != cudaSuccess) return GG_ERR_CUDA;
  void* buf = c->hdri;
  int st = grow(&buf, &c->hdri_cap, bytes);
  c->hdri = static_cast<float*>(buf);
  if (st != GG_OK) return st;
  // on the context's (non-blocking) stream and waited for: a copy from
  // pageable memory may otherwise return before it has landed
  if (cudaMemcpyAsync(c->hdri, rgb, bytes, cudaMemcpyHostToDevice, c->stream) != cudaSuccess ||
      cudaStreamSynchronize(c->stream) != cudaSuccess)
    return GG_ERR_CUDA;
  c->hdri_w = width;
  c->hdri_h = height;
  c->hdri_intensity = intensity;
  return GG_OK;
}

GG_API int gg_set_scene(gg_ctx* c, const gg_prim_t* prims, uint32_t n) {
  if (!c) return GG_ERR_INVALID_ARG;
  std::vector<gg::ScenePrim> ps;
  std::vector<gg::SceneNode> nodes;
  if (n > 0) {
    const int st = gg::build_scene(prims, n, &ps, &nodes, nullptr);
    if (st != GG_OK) return st;
  }
  Lock lock(c);
  // renders in flight may read the old scene
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) return GG_ERR_CUDA;
  if (cudaEventSynchronize(c->ev_done) != cudaSuccess) return GG_ERR_CUDA;
  c->scene_set = false;
  if (n == 0) return GG_OK;
  const size_t pb = ps.size() * sizeof(gg::ScenePrim), nb = nodes.size() * sizeof(gg::SceneNode);
  int st = grow(&c->scene_prims, &c->scene_prims_cap, pb);
  if (st != GG_OK) return st;
  st = grow(&c->scene_nodes, &c->scene_nodes_cap, nb);
  if (st != GG_OK) return st;
  if (cudaMemcpyAsync(c->scene_prims, ps.data(), pb, cudaMemcpyHostToDevice, c->stream) !=
          cudaSuccess ||
      cudaMemcpyAsync(c->scene_nodes, nodes.data(), nb, cudaMemcpyHostToDevice, c->stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(c->stream) != cudaSuccess)
    return GG_ERR_CUDA;
  c->scene_set = true;
  return GG_OK;
}

GG_API int gg_scene_validate(const gg_prim_t* prims, uint32_t n, uint32_t* n_nodes,
                             uint32_t* depth) {
  std::vector<gg::ScenePrim> ps;
  std::vector<gg::SceneNode> nodes;
  const int st = gg::build_scene(prims, n, &ps, &nodes, depth);
  if (st == GG_OK && n_nodes) *n_nodes = (uint32_t)nodes.size();
  return st;
}

GG_API int gg_batch_variant_info(int v, int32_t out[4]) {
  if (!out || v < 0 || v >= GG_BATCH_VARIANTS) return GG_ERR_INVALID_ARG;
  const gg::BatchVariant& b = gg::kBatchVariantTable[v];
  out[0] = b.period;
  out[1] = b.ctas_per_sm;
  out[2] = b.block;
  out[3] = b.chunk;
  return GG_OK;
}

GG_API int gg_batch_set_variant(gg_ctx* c, int variant) {
  if (!c || variant < 0 || variant >= GG_BATCH_VARIANTS) return GG_ERR_INVALID_ARG;
  Lock lock(c);
  c->batch_variant = variant;
  return GG_OK;
}

GG_API int gg_forward_ckpt(gg_ctx* c, const gg_metric_t* metric, double r_cam,
                           double inclination, double fov_y_radians, double aspect,
                           const gg_disk_t* disk, const gg_integrator_t* integ,
                           const gg_render_opts_t* opts, uint32_t width, uint32_t height,
                           double* rgb_lin_dev, void* stream) {
  if (!c || !metric || !disk || !integ || !opts || !rgb_lin_dev) return GG_ERR_INVALID_ARG;
  gg_camera_t cam;
  if (gg_camera_inclined(&cam, r_cam, inclination, fov_y_radians, aspect) != GG_OK)
    return GG_ERR_INVALID_ARG;
  const int v = validate(metric, &cam, disk, integ, opts, width, height);
  if (v != GG_OK) return v;
  if (metric->kind != GG_METRIC_KERR || disk->kind != GG_DISK_THIN ||
      integ->precision != GG_PREC_FP64 || integ->stepper != GG_STEPPER_DP45 ||
      opts->samples_per_axis > 1 || opts->jitter_spp > 0 || opts->attempt_budget != 0 ||
      opts->sky == GG_SKY_HDRI || opts->scene)
    return GG_ERR_UNSUPPORTED;
  Lock lock(c);
  DevParams P;
  build_params(metric, &cam, disk, integ, opts, width, height, &P);
  P.ckpt = 1;
  const uint32_t cpr = integ->max_steps / gg::kCkptEvery + 2;
  int st = grow(&c->diff_rays, &c->diff_rays_cap, sizeof(gg::DiffRay) * P.n_rays);
  if (st != GG_OK) return st;
  st = grow(&c->diff_ckpt, &c->diff_ckpt_cap, sizeof(gg::Ckpt) * cpr * P.n_rays);
  if (st != GG_OK) return st;
  // the FP64 trace kernel's checkpointing variant: linear colour per ray,
  // checkpoints and DiffRay
  DevOutputs O{};
  O.rgb = rgb_lin_dev;
  O.ckpt = static_cast<gg::Ckpt*>(c->diff_ckpt);
  O.diff_rays = static_cast<gg::DiffRay*>(c->diff_rays);
  O.ckpt_per_ray = cpr;
  c->diff_ready = false;
  st = enqueue(c, P, O, false, static_cast<cudaStream_t>(stream));
  if (st != GG_OK) return st;
  c->diff_P = P;
  c->diff_ckpt_per_ray = cpr;
  c->diff_ready = true;
  return GG_OK;
}

GG_API int gg_backward(gg_ctx* c, const double* dl_drgb_dev, double grad[5], void* stream) {
  if (!c || !dl_drgb_dev || !grad) return GG_ERR_INVALID_ARG;
  Lock lock(c);
  if (!c->diff_ready) return GG_ERR_INVALID_ARG;
  if (!c->diff_grad && cudaMalloc(&c->diff_grad, 5 * sizeof(double)) != cudaSuccess) {
    cudaGetLastError();
    c->diff_grad = nullptr;
    return GG_ERR_OOM;
  }
  if (!c->diff_grad_host &&
      cudaMallocHost(&c->diff_grad_host, 5 * sizeof(double)) != cudaSuccess) {
    cudaGetLastError();
    c->diff_grad_host = nullptr;
    return GG_ERR_OOM;
  }
  const int gl = grow(&c->diff_list, &c->diff_list_cap,
                     gg::backward_list_bytes(c->diff_P.n_rays, c->diff_ckpt_per_ray));
  if (gl != GG_OK) return gl;
  gg::DiffOut D{static_cast<gg::DiffRay*>(c->diff_rays), static_cast<gg::Ckpt*>(c->diff_ckpt),
                c->diff_ckpt_per_ray, 0u};
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (cudaStreamWaitEvent(s, c->ev_done, 0) != cudaSuccess) return GG_ERR_CUDA;
  if (cudaMemsetAsync(c->diff_grad, 0, 5 * sizeof(double), s) != cudaSuccess) return GG_ERR_CUDA;
  if (gg::launch_diff_backward(c->diff_P, D, dl_drgb_dev, c->diff_grad, c->diff_list, c->sms,
                               s) != cudaSuccess)
    return GG_ERR_CUDA;
  if (cudaMemcpyAsync(c->diff_grad_host, c->diff_grad, 5 * sizeof(double),
                      cudaMemcpyDeviceToHost, s) != cudaSuccess)
    return GG_ERR_CUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return GG_ERR_CUDA;
  for (int i = 0; i < 5; ++i) grad[i] = c->diff_grad_host[i];
  cudaEventRecord(c->ev_done, s);
  return GG_OK;
}

GG_API int gg_render(gg_ctx* c, const gg_metric_t* metric, const gg_camera_t* camera,
                     const gg_disk_t* disk, const gg_integrator_t* integ,
                     const gg_render_opts_t* opts, uint32_t width, uint32_t height,
                     uint8_t* rgb_out, const gg_ray_out_t* rays_out) {
  if (!c) return GG_ERR_INVALID_ARG;
  const int v = validate(metric, camera, disk, integ, opts, width, height);
  if (v != GG_OK) return v;
  const int sup = supported(disk, integ, opts);
  if (sup != GG_OK) return sup;
  DevParams P;
  build_params(metric, camera, disk, integ, opts, width, height, &P);
  Lock lock(c);
  const int sky = attach_sky_map(c, &P);
  if (sky != GG_OK) return sky;
  const uint64_t n = P.n_rays;
  const size_t n_pix = (size_t)width * P.rows;

  // lay out the device staging buffer for every requested output
  struct Slot {
    void* host;
    size_t bytes;
    size_t off;
  };
  Slot slots[11];
  int ns = 0;
  size_t total = 0;
  auto add = [&](void* host, size_t bytes) -> size_t {
    if (!host) return (size_t)-1;
    slots[ns] = {host, bytes, total};
    ++ns;
    const size_t off = total;
    total += align256(bytes);
    return off;
  };
  const size_t o_rgb8 = add(rgb_out, n_pix * 3);
  size_t o_arr[10];
  for (int k = 0; k < 10; ++k) o_arr[k] = (size_t)-1;
  if (rays_out) {
    o_arr[0] = add(rays_out->cls, n * sizeof(int32_t));
    o_arr[1] = add(rays_out->x, n * 4 * sizeof(double));
    o_arr[2] = add(rays_out->v, n * 4 * sizeof(double));
    o_arr[3] = add(rays_out->lambda, n * sizeof(double));
    o_arr[4] = add(rays_out->attempts, n * sizeof(uint32_t));
    o_arr[5] = add(rays_out->accepted, n * sizeof(uint32_t));
    o_arr[6] = add(rays_out->intensity, n * sizeof(double));
    o_arr[7] = add(rays_out->color_temp, n * sizeof(double));
    o_arr[8] = add(rays_out->rgb, n * 3 * sizeof(double));
    o_arr[9] = add(rays_out->cross, n * 8 * sizeof(double));
  }
  if (total > 0) {
    const int st = grow(&c->staging, &c->staging_cap, total);
    if (st != GG_OK) return st;
  }
  char* base = static_cast<char*>(c->staging);
  auto dp = [&](size_t off) -> void* { return off == (size_t)-1 ? nullptr : base + off; };
  DevOutputs O;
  std::memset(&O, 0, sizeof(O));
  O.rgb8 = static_cast<uint8_t*>(dp(o_rgb8));
  O.cls = static_cast<int32_t*>(dp(o_arr[0]));
  O.x = static_cast<double*>(dp(o_arr[1]));
  O.v = static_cast<double*>(dp(o_arr[2]));
  O.lam = static_cast<double*>(dp(o_arr[3]));
  O.attempts = static_cast<uint32_t*>(dp(o_arr[4]));
  O.accepted = static_cast<uint32_t*>(dp(o_arr[5]));
  O.intensity = static_cast<double*>(dp(o_arr[6]));
  O.color_temp = static_cast<double*>(dp(o_arr[7]));
  O.rgb = static_cast<double*>(dp(o_arr[8]));
  O.cross = static_cast<double*>(dp(o_arr[9]));

  int st = enqueue(c, P, O, rgb_out != nullptr, c->stream);
  if (st != GG_OK) return st;
  for (int k = 0; k < ns; ++k) {
    if (cudaMemcpyAsync(slots[k].host, base + slots[k].off, slots[k].bytes,
                        cudaMemcpyDeviceToHost, c->stream) != cudaSuccess)
      return GG_ERR_CUDA;
  }
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) return GG_ERR_CUDA;
  return collect(c);
}

}  // extern "C"
