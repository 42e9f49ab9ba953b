// gg_params.h -- the launch-time parameter block of the trace kernels.
//
// Built once per render on the host from the public POD structs.  Every
// per-render constant that the reference recomputes per ray (the camera's
// orthonormal frame, tan(fov/2), the metric at the camera, the observer's
// -g_tt) is evaluated here on the host in the reference's operation order,
// so the kernels only do per-sample arithmetic.  Passed by value as a
// __grid_constant__ kernel parameter (uniform across the grid).
#pragma once

#include <cstdint>

namespace gg {

enum : int { kMetricSchwarzschild = 0, kMetricKerr = 1 };
enum : int { kDiskNone = 0, kDiskVolumetric = 1, kDiskThin = 2 };
enum : int { kSkyProcedural = 0, kSkyChecker = 1, kSkyHdri = 2 };
enum : int {
  kClsHorizon = 0,
  kClsEscaped = 1,
  kClsDisk = 2,
  kClsMaxSteps = 3,
  kClsBudget = 4,
  kClsScene = 5,
  kNumClasses = 6
};

// Scene primitive with the quantities its hit test and shading read,
// prepared on the host: Sphere (sphere.rs:53-87), Quad (quad.rs:36-125,
// with its precomputed unit normal, plane offset and e_alpha / e_beta).
enum : int { kPrimSphere = 0, kPrimQuad = 1 };
// shade_hit's albedo (tracer.rs:369-384): the material's scatter attenuation
// when it scatters -- always (Lambertian, Dielectric: white), never
// (DiffuseLight), or when the mirror direction leaves the surface (Metal
// with fuzz 0).
enum : int { kShadeAlbedo = 0, kShadeEmit = 1, kShadeMirror = 2 };
struct ScenePrim {
  int kind, shade;
  double c[3];  // sphere centre / quad corner
  double radius;
  double n[3];  // quad unit normal
  double d;     // quad plane offset n . Q
  double ea[3], eb[3];
  double albedo[3], emit[3];
};
// Bounding-volume hierarchy node: count > 0 is a leaf over prims
// [first, first + count); count == 0 an inner node with children first and
// first + 1.
struct SceneNode {
  double lo[3], hi[3];
  int first, count;
};
constexpr int kSceneStack = 64;  // traversal stack; the host caps the depth below it
enum : int { kStepperReference = 0, kStepperDP45 = 1 };

struct DevParams {
  // metric
  int metric;
  int has_horizon;
  double mass, spin, rs;
  double rh, rh_plus_buffer;
  double r_photon;  // prograde circular photon orbit (mixed form's FP64 band)
  // integrator
  double initial_step, min_step, max_step, tolerance, max_radius;
  double rtol, atol;
  uint32_t max_steps;
  int precision;
  int stepper;
  int pad_stepper;
  // mixed form: FP32 copies of the constants its stepping loop reads, and the
  // FP64 band -- an attempt that starts at r < band_r, or with theta within
  // pole_band of a pole, is handed to the FP64 pass
  float mass_f, spin_f, rs_f, atol_f, rtol_f;
  float max_radius_hi, max_radius_lo;  // max_radius as an unevaluated float pair
  float band_r, pole_band;
  // FP64 pass over the band queue: return a ray to the mixed form (the
  // O.ret queue) once it is clear of the band (gg_trace.cu, kBackMargin)
  uint32_t hand_back;
  // the FP32 Kerr right-hand side's per-render constants: a^2, 2M, -2a^2,
  // 2Ma, 4Ma, 2Ma^2, 4Ma^2
  float a2_f, m2_f, mm2a2_f, m2a_f, m4a_f, m2a2_f, m4a2_f;
  // sampling
  uint32_t width, height, spa, spp, jitter_spp, sub_w, sub_h;
  uint32_t pad0;
  uint32_t row0, row_step, rows;  // traced rows: row0 + k row_step, k < rows
  uint32_t pad_rows;
  uint64_t seed;
  uint64_t n_rays;
  // camera frame (camera.rs:20-29, ray.rs:29-48), host-evaluated
  double cam_pos[4];
  double cam_forward[3], cam_right[3], cam_up[3];
  double half_w, half_h;
  double r_hat[3], theta_hat[3], phi_hat[3];
  double cam_g_tt, cam_g_rr, cam_g_thth, cam_g_phph;
  double sqrt_g_rr, sqrt_g_thth, sqrt_g_phph;
  double sqrt_neg_gtt_obs;  // tracer.rs:93-94
  // disk
  int disk;
  int pad1;
  double r_inner, r_outer, scale_height, density_0, temperature_0, emissivity_index;
  // sky
  int sky;
  uint32_t sky_rows, sky_cols;
  uint32_t pad2;
  uint64_t sky_seed;
  double cell_h, cell_w;
  const float* hdri;  // GG_SKY_HDRI: the context's map, hdri_w x hdri_h RGB texels
  uint32_t hdri_w, hdri_h;
  float hdri_intensity;
  float pad_hdri;
  // opts.scene: the context's scene, its hierarchy rooted at nodes[0]
  const ScenePrim* prims;
  const SceneNode* nodes;
  uint32_t scene;
  // gg_forward_ckpt: the FP64 kernel also stores each ray's checkpoints and
  // DiffRay (DevOutputs::ckpt, diff_rays)
  uint32_t ckpt;
  // control
  uint64_t attempt_budget;
  double inv_spp;
};

// Device pointers of one render's outputs (each nullable).
struct DevOutputs {
  int32_t* cls;
  double* x;
  double* v;
  double* lam;
  uint32_t* attempts;
  uint32_t* accepted;
  double* intensity;
  double* color_temp;
  double* rgb;
  double* cross;
  uint8_t* rgb8;        // image, written directly when spp == 1
  double* sample_rgb;   // 3*n linear sample colours, reduced per pixel when spp > 1
  struct QueuedRay* queue;  // mixed form: rays handed to the FP64 pass
  uint64_t queue_cap;
  struct QueuedRay* ret;    // mixed form: rays the FP64 pass hands back
  uint64_t ret_cap;
  struct Ckpt* ckpt;         // differentiable render: ckpt_per_ray entries per ray
  struct DiffRay* diff_rays;
  uint32_t ckpt_per_ray;
  uint32_t pad_ckpt;
};

// A ray the mixed-precision pass hands to the FP64 pass (its state at the
// start of the attempt that entered the FP64 band) or the FP64 pass hands
// back (its state after the step that left the band), in FP64.
struct QueuedRay {
  double x[4];
  double v[4];
  double h;
  double lam;
  uint64_t idx;  // sample index (within its scene)
  uint32_t n_att, n_acc;
  uint32_t scene;  // batched renders: the ray's scene
  uint32_t pad;
};

// One scene of a batched render: its parameters (camera, metric, disk, sky,
// image size; the integrator is the batch's) and its output pointers.
struct BatchScene {
  DevParams P;
  DevOutputs O;
};

// Differentiable render (gg_forward_ckpt / gg_backward): what the forward
// pass keeps per ray for the backward pass.
struct DiffRay {
  uint32_t n_acc;   // accepted steps
  uint32_t n_ckpt;  // checkpoints stored; the first is the initial state
  int32_t cls;
  uint32_t pad;
};
// Accepted steps between checkpoints of the differentiable render's forward.
constexpr int kCkptEvery = 32;
struct Ckpt {  // state after every kCkptEvery-th accepted step, and the next step size
  double x[4];
  double v[4];
  double h;
};
struct DiffOut {  // what the backward pass reads
  DiffRay* rays;
  Ckpt* ckpt;          // ckpt_per_ray entries per ray
  uint32_t ckpt_per_ray;
  uint32_t pad;
};

// Where a batched launch finds its scenes: first[k] is the global index of
// scene k's first sample (first[n] = total samples).
struct BatchTable {
  const BatchScene* scenes;
  const uint64_t* first;
  uint32_t n;
  uint32_t pad;
};

// Device-side counters of one render (reset before each launch).
struct DevControl {
  unsigned long long next_ray;   // work queue head
  unsigned long long attempts;   // step() calls, all rays
  unsigned long long accepted;
  unsigned long long class_count[kNumClasses];
  unsigned long long budget_used;
  unsigned int abort;            // set once the attempt budget is spent
  unsigned int queue_overflow;   // a mixed-form hand-off found the queue full
  unsigned long long queued;     // rays handed to the FP64 pass
  unsigned long long next_queued;  // the FP64 pass's queue head
  unsigned long long fp64_attempts;  // attempts made in the FP64 pass
  unsigned long long returned;       // rays the FP64 pass handed back to the mixed form
  unsigned long long next_returned;  // the mixed form's head on that queue
  unsigned long long band_total;     // hand-offs to the FP64 pass of earlier rounds
};

}  // namespace gg
