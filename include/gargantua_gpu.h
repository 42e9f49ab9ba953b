/*
 * gargantua_gpu.h -- C ABI of the B200 (sm_100a) general-relativistic ray path.
 *
 * The library renders images of a Schwarzschild or Kerr black hole by
 * integrating one null geodesic per image sample on the GPU with the
 * gargantua RK45 (Dormand-Prince) stepper, ends each ray at the horizon, the
 * accretion disk or the escape sphere, and shades it.  Every entry point is
 * plain C: POD structs, raw pointers and sizes, an int status.  No call
 * aborts, panics or traps; failures come back as a negative status.
 *
 * Reference interface each group replaces (paths are inside gargantua):
 *   gg_metric_*        gr-core  Metric impls   crates/gr-core/src/schwarzschild.rs:12-23,
 *                                              crates/gr-core/src/kerr.rs:24-34
 *   gg_integrator_*    gr-core  RK45Integrator crates/gr-core/src/geodesic.rs:155-181
 *                      plus the renderer's overrides
 *                                              crates/raytracer/src/curved/renderer.rs:264-265
 *   gg_camera_t        raytracer::curved::Camera crates/raytracer/src/curved/camera.rs:9-15
 *   gg_disk_t          raytracer::curved::AccretionDisk crates/raytracer/src/curved/disk.rs:8-31
 *   gg_render          raytracer::curved::render / render_with_disk
 *                                              crates/raytracer/src/curved/renderer.rs:82-101
 *   gg_ray_out_t       raytracer::curved::RayOutcome crates/raytracer/src/curved/outcome.rs:4-22
 *                      plus the final GeodesicState crates/gr-core/src/geodesic.rs:13-30
 *
 * Threading: one gg_ctx per host thread.  A context owns one CUDA stream and
 * the device scratch it grows on demand; calls on one context are serialised.
 */
#ifndef GARGANTUA_GPU_H
#define GARGANTUA_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define GG_API __attribute__((visibility("default")))
#else
#define GG_API
#endif

/* ---- status codes ------------------------------------------------------ */
#define GG_OK 0
#define GG_ERR_INVALID_ARG (-1) /* a parameter fails validation            */
#define GG_ERR_CUDA (-2)        /* a CUDA runtime call failed              */
#define GG_ERR_OOM (-3)         /* device allocation failed                */
#define GG_ERR_BUDGET (-4)      /* the attempt budget ran out mid-render   */
#define GG_ERR_UNSUPPORTED (-5) /* combination not implemented             */
#define GG_ERR_NO_DEVICE (-6)   /* no CUDA device / not an sm_100 device   */
#define GG_ERR_TOO_LARGE (-7)   /* beyond gg_render_device_noalloc's fixed scratch */

/* ---- metric (gr-core Metric implementations) --------------------------- */
#define GG_METRIC_SCHWARZSCHILD 0
#define GG_METRIC_KERR 1

typedef struct gg_metric_t {
  int32_t kind;  /* GG_METRIC_* */
  int32_t reserved;
  double mass;   /* M > 0 */
  double spin;   /* Kerr a, clamped to |a| <= 0.9999 M by gg_metric_kerr */
} gg_metric_t;

/* ---- camera (raytracer::curved::Camera) -------------------------------- */
typedef struct gg_camera_t {
  double position[4]; /* (t, r, theta, phi) in the metric's chart          */
  double look_at[3];  /* local Cartesian frame, projected on r,theta,phi    */
  double up[3];
  double fov_y_radians;
  double aspect;      /* width / height of the image plane                  */
} gg_camera_t;

/* ---- accretion disk ---------------------------------------------------- */
#define GG_DISK_NONE 0       /* render(): trace_ray                            */
#define GG_DISK_VOLUMETRIC 1 /* render_with_disk(): Gaussian volumetric disk   */
#define GG_DISK_THIN 2       /* thin equatorial disk, emissivity (r_in/r)^q    */

typedef struct gg_disk_t {
  int32_t kind; /* GG_DISK_* */
  int32_t reserved;
  double r_inner;
  double r_outer;
  double scale_height;     /* volumetric: Gaussian H                        */
  double density_0;        /* volumetric: rho_0                             */
  double temperature_0;    /* volumetric: reported colour temperature       */
  double emissivity_index; /* thin: q in I_emit = (r_inner / r)^q           */
} gg_disk_t;

/* ---- integrator (gr-core RK45Integrator + renderer loop bound) ---------- */
#define GG_PREC_FP64 0  /* plain FP64, the drop-in                           */
#define GG_PREC_MIXED 1 /* FP32 stages + compensated state, FP64 controller  */

/* The reference's RK45Integrator::step (geodesic.rs:185-328) moves the
 * position by h * vel (first order) and controls the velocity error only.
 * GG_STEPPER_DP45 is the full Dormand-Prince RK5(4) on (x, v): positions
 * from the stage velocities, error control over all eight components, the
 * reference's termination tests and step-size law, crossings located on the
 * pair's 4th-order continuous extension (dense output). */
#define GG_STEPPER_REFERENCE 0
#define GG_STEPPER_DP45 1

typedef struct gg_integrator_t {
  double initial_step;
  double min_step;
  double max_step;
  double tolerance;      /* absolute velocity-error tolerance (rtol == 0)    */
  double max_radius;     /* escape radius                                    */
  double horizon_buffer; /* Horizon when r < r_h + horizon_buffer            */
  double rtol;           /* > 0: scaled error norm, atol + rtol*max(|v|,|v'|) */
  double atol;
  uint32_t max_steps;    /* step() calls per ray before MaxSteps             */
  int32_t precision;     /* GG_PREC_*                                        */
  int32_t stepper;       /* GG_STEPPER_*                                     */
  int32_t reserved;
} gg_integrator_t;

/* ---- render options (raytracer::curved::RenderOptions) ----------------- */
#define GG_SKY_PROCEDURAL 0 /* hashed starfield over a blue gradient          */
#define GG_SKY_CHECKER 1    /* seeded checkerboard over (theta, phi) cells     */
#define GG_SKY_HDRI 2       /* equirectangular map of the context (gg_set_hdri) */

typedef struct gg_render_opts_t {
  uint32_t samples_per_axis; /* stratified supersampling, spa*spa per pixel */
  uint32_t jitter_spp;       /* 0: stratified; n>0: n seeded uniform offsets */
  uint64_t seed;             /* jitter seed                                 */
  int32_t sky;               /* GG_SKY_*                                    */
  uint32_t sky_rows;         /* checkerboard cells in theta (18)            */
  uint32_t sky_cols;         /* checkerboard cells in phi (36)              */
  uint32_t row_offset;       /* with row_step: first image row traced       */
  uint64_t sky_seed;
  uint64_t attempt_budget;   /* 0: unlimited; else GG_ERR_BUDGET past it    */
  /* row_step > 1: trace only image rows row_offset, row_offset + row_step,
   * ... (one GPU's share of a frame split across GPUs, interleaved so every
   * share gets rows through the shadow); the image and per-sample outputs
   * then hold those rows only, in order.  0 or 1: every row. */
  uint32_t row_step;
  /* 1: test every step's straight chord against the context's scene
   * (gg_set_scene), render_with_scene / render_with_disk_and_scene
   * (crates/raytracer/src/curved/renderer.rs:110-254); 0: no scene. */
  uint32_t scene;
} gg_render_opts_t;

/* ---- per-sample outcome (RayOutcome + final GeodesicState) ------------- */
#define GG_CLASS_HORIZON 0
#define GG_CLASS_ESCAPED 1
#define GG_CLASS_DISK 2
#define GG_CLASS_MAXSTEPS 3
#define GG_CLASS_BUDGET 4 /* not traced: the attempt budget ran out         */
#define GG_CLASS_SCENE 5  /* a step's chord hit the scene (RayOutcome::Scene) */
#define GG_N_CLASSES 6

/* Every pointer is optional (NULL: not written).  Arrays have one entry per
 * sample, ordered sample-major inside a pixel and pixels row-major:
 * index = (py * width + px) * spp + s, with spp = spa*spa (s = sy*spa + sx)
 * or jitter_spp.  x and v are component-major: x[c * n + i]. */
typedef struct gg_ray_out_t {
  int32_t* cls;        /* GG_CLASS_*                                      */
  double* x;           /* 4*n final position (t, r, theta, phi)           */
  double* v;           /* 4*n final velocity (dt, dr, dtheta, dphi)/dlam  */
  double* lambda;      /* n affine parameter                              */
  uint32_t* attempts;  /* n step() calls                                  */
  uint32_t* accepted;  /* n accepted steps                                */
  double* intensity;   /* n disk intensity (0 if none)                    */
  double* color_temp;  /* n disk colour temperature (0 if none)           */
  double* rgb;         /* 3*n linear colour of the sample, interleaved    */
  double* cross;       /* 8*n state (x, v) where the ray met the escape
                        * sphere r = max_radius or the thin disk plane,
                        * interpolated on the last accepted step; NaN for
                        * rays that ended elsewhere; component-major       */
} gg_ray_out_t;

/* ---- statistics of the last render on a context ------------------------ */
typedef struct gg_stats_t {
  uint64_t rays;
  uint64_t attempts;
  uint64_t accepted;
  uint64_t class_count[GG_N_CLASSES];
  double kernel_ms; /* device time of the trace launch(es)                 */
  /* GG_PREC_MIXED: rays the FP32 pass handed to the FP64 pass (FP64 band)
   * and the attempts made in that pass; 0 for GG_PREC_FP64 */
  uint64_t fp64_rays;
  uint64_t fp64_attempts;
} gg_stats_t;

typedef struct gg_ctx gg_ctx;

/* ---- library ----------------------------------------------------------- */
GG_API const char* gg_version(void);
GG_API const char* gg_strerror(int status);
/* sizeof of a public struct by name ("gg_metric_t", ...), -1 if unknown */
GG_API int gg_struct_size(const char* name);

/* ---- parameter constructors (host only, no device work) ---------------- */
/* Schwarzschild::new(mass) (schwarzschild.rs:13-18) */
GG_API int gg_metric_schwarzschild(gg_metric_t* out, double mass);
/* Kerr::new(mass, spin) (kerr.rs:29-34): mass <= 0 is GG_ERR_INVALID_ARG
 * where the reference asserts; spin is clamped to +-0.9999 mass. */
GG_API int gg_metric_kerr(gg_metric_t* out, double mass, double spin);
/* RK45Integrator::default() (geodesic.rs:170-181) with the renderer's
 * max_radius = 200 and max_steps = 5000 (renderer.rs:264-265). */
GG_API void gg_integrator_default(gg_integrator_t* out);
/* AccretionDisk::default() (disk.rs:21-31) as a volumetric disk. */
GG_API void gg_disk_default(gg_disk_t* out);
/* RenderOptions::default() with samples_per_axis = 1 (renderer.rs:267). */
GG_API void gg_render_opts_default(gg_render_opts_t* out);
/* Pinhole camera at (0, r, incl, 0) looking at the hole, up = +z. */
GG_API int gg_camera_inclined(gg_camera_t* out, double r, double inclination_rad,
                              double fov_y_radians, double aspect);
/* Prograde ISCO (Bardeen-Press-Teukolsky) and prograde circular photon
 * orbit radii of a Kerr hole; a = 0 gives 6M and 3M. */
GG_API double gg_kerr_isco(double mass, double spin);
GG_API double gg_kerr_photon_orbit(double mass, double spin);
/* Checks every field a render would use; GG_OK or GG_ERR_INVALID_ARG. */
GG_API int gg_validate(const gg_metric_t* metric, const gg_camera_t* camera,
                       const gg_disk_t* disk, const gg_integrator_t* integ,
                       const gg_render_opts_t* opts, uint32_t width, uint32_t height);

/* ---- context ----------------------------------------------------------- */
GG_API int gg_create(gg_ctx** out, int device);
GG_API int gg_destroy(gg_ctx* ctx);
/* The context's CUDA stream (a cudaStream_t). */
GG_API void* gg_stream(gg_ctx* ctx);
GG_API int gg_last_stats(gg_ctx* ctx, gg_stats_t* out);

/* ---- rendering --------------------------------------------------------- */
/* Drop-in for render / render_with_disk (renderer.rs:82-101).  Synchronous.
 * rgb_out: host, width*height*3 bytes row-major (RgbImage layout), may be
 * NULL.  rays_out: host arrays, may be NULL.  disk may be NULL (no disk). */
GG_API int gg_render(gg_ctx* ctx, const gg_metric_t* metric, const gg_camera_t* camera,
                     const gg_disk_t* disk, const gg_integrator_t* integ,
                     const gg_render_opts_t* opts, uint32_t width, uint32_t height,
                     uint8_t* rgb_out, const gg_ray_out_t* rays_out);

/* Same render with DEVICE output pointers, enqueued on `stream` (a
 * cudaStream_t; NULL is CUDA's default stream; gg_stream(ctx) gives the
 * context's own) without synchronising.  Scratch comes from the context;
 * gg_last_stats waits for this render. */
GG_API int gg_render_device(gg_ctx* ctx, const gg_metric_t* metric, const gg_camera_t* camera,
                            const gg_disk_t* disk, const gg_integrator_t* integ,
                            const gg_render_opts_t* opts, uint32_t width, uint32_t height,
                            uint8_t* rgb_dev, const gg_ray_out_t* rays_dev, void* stream);

/* For callers that must not let a library allocate device memory (their
 * own arena or pool owns every byte, or allocation after start-up is
 * forbidden, or a cudaMalloc's device-wide synchronisation is unacceptable).
 * No counterpart in the reference, which has no device code.
 *
 * Same render as gg_render_device, but without a context and without any
 * allocation: it calls no cudaMalloc / cudaFree and no allocating library
 * routine.  Its scratch (work-queue counters and, when samples_per_axis > 1
 * or jitter_spp > 1, one linear colour per sample) is a 16 MiB array that
 * every GPU which loads this library holds until the process exits.
 *   - Works on the current device; outputs are device pointers; enqueued on
 *     `stream` (NULL = CUDA's default stream) without synchronising.
 *   - Supersampled images are limited to 699,040 samples
 *     (width * height * spp); larger ones return GG_ERR_TOO_LARGE.
 *     Single-sample images have no size limit here.
 *   - Every call looks up the array's device address in the current
 *     context, so the entry point stays valid after cudaDeviceReset and
 *     under any context.  The first call on a device also loads this
 *     library's device code there: make that first call before any stream
 *     capture.
 *   - Every call on a device shares the one array: calls whose work overlaps
 *     on the GPU (different streams, not ordered) race and corrupt each
 *     other's results.  Order them, for example on one stream.
 *   - The attempt budget and the mixed precision form are not offered here
 *     (GG_ERR_UNSUPPORTED); no statistics are returned. */
GG_API int gg_render_device_noalloc(const gg_metric_t* metric, const gg_camera_t* camera,
                                    const gg_disk_t* disk, const gg_integrator_t* integ,
                                    const gg_render_opts_t* opts, uint32_t width,
                                    uint32_t height, uint8_t* rgb_dev,
                                    const gg_ray_out_t* rays_dev, void* stream);

/* ---- batched rendering (no reference counterpart) ---------------------- */
/* One scene of a batch: its own metric, camera, disk, image size and sky
 * seed.  The integrator and render options are the batch's. */
typedef struct gg_scene_t {
  gg_metric_t metric;
  gg_camera_t camera;
  gg_disk_t disk;    /* GG_DISK_NONE or GG_DISK_THIN, one kind per batch     */
  uint32_t width;
  uint32_t height;
  uint64_t sky_seed; /* checkerboard seed of this scene                      */
} gg_scene_t;

#define GG_BATCH_VARIANTS 12 /* kernel variants the batch autotuner chooses from */

/* Renders n scenes in one persistent launch of the mixed-precision kernel
 * (integ: GG_PREC_MIXED, GG_STEPPER_DP45; opts: one sample per pixel), its
 * FP64 band pass after it.  All scenes share one metric kind and one disk
 * kind.  The launch sequence is captured in a CUDA graph per batch shape
 * (scene count, total samples, integrator and options) and replayed; the
 * scenes' parameters are uploaded from the context's pinned buffer by a copy
 * node inside the graph, so a batch of the same shape with new cameras,
 * spins or disks reuses the graph.  The kernel variant (compaction period,
 * register budget, threads per CTA and samples per work-queue claim; see
 * gg_batch_variant_info) is the one gg_batch_autotune chose on this context,
 * or a fixed default.
 * gg_render_batch_device: images concatenated in scene order into rgb_dev
 * (scene k at byte 3 * sum_{j<k} w_j h_j), enqueued on `stream` (NULL = CUDA's
 * default stream).  gg_render_batch: synchronous, rgb_out[k] = scene k's
 * host buffer of w_k * h_k * 3 bytes.  Statistics via gg_last_stats. */
GG_API int gg_render_batch_device(gg_ctx* ctx, const gg_scene_t* scenes, uint32_t n,
                                  const gg_integrator_t* integ, const gg_render_opts_t* opts,
                                  uint8_t* rgb_dev, void* stream);
GG_API int gg_render_batch(gg_ctx* ctx, const gg_scene_t* scenes, uint32_t n,
                           const gg_integrator_t* integ, const gg_render_opts_t* opts,
                           uint8_t* const* rgb_out);
/* Times each of the GG_BATCH_VARIANTS kernel variants on this batch (one
 * render each, images discarded), keeps the fastest for the context's later
 * batches and returns its index; ms_out (nullable, GG_BATCH_VARIANTS entries)
 * receives each variant's device time. */
GG_API int gg_batch_autotune(gg_ctx* ctx, const gg_scene_t* scenes, uint32_t n,
                             const gg_integrator_t* integ, const gg_render_opts_t* opts,
                             int* variant_out, double* ms_out);
/* Sets the context's batch kernel variant (0 .. GG_BATCH_VARIANTS-1). */
GG_API int gg_batch_set_variant(gg_ctx* ctx, int variant);
/* The settings of batch kernel variant v: out[0] refill period (attempts
 * between a warp's refills), out[1] CTAs per SM its registers are budgeted
 * for, out[2] threads per CTA, out[3] samples a warp claims from the work
 * queue at a time.  0, or GG_ERR_INVALID_ARG.  Host only; no device needed. */
GG_API int gg_batch_variant_info(int v, int32_t out[4]);

/* ---- differentiable render (no reference counterpart) ------------------- */
/* Forward pass of the differentiable render: Kerr (metric), the inclined
 * camera gg_camera_inclined(r_cam, inclination, fov_y, aspect), a thin disk,
 * integ GG_PREC_FP64 + GG_STEPPER_DP45, opts one sample per pixel and no
 * budget.  Writes the linear RGB image (width*height*3 doubles, row-major,
 * device pointer) on `stream` and keeps, in the context, per-ray
 * checkpoints of the state every 32 accepted steps for gg_backward.
 * With opts->row_step > 1 only the rows row_offset, row_offset + row_step,
 * ... are traced and the image holds those rows, in order (one rank's share
 * of a data-parallel gradient: the ranks' gg_backward results add up to the
 * whole image's).  The image is a function of p = (spin, inclination, r_cam,
 * disk r_inner, disk emissivity_index). */
GG_API int gg_forward_ckpt(gg_ctx* ctx, const gg_metric_t* metric, double r_cam,
                           double inclination, double fov_y_radians, double aspect,
                           const gg_disk_t* disk, const gg_integrator_t* integ,
                           const gg_render_opts_t* opts, uint32_t width, uint32_t height,
                           double* rgb_lin_dev, void* stream);
/* Adjoint of the last gg_forward_ckpt on this context: given dL/d(image)
 * (device, same layout), writes dL/dp to grad[5] (host) in the order above.
 * Disk pixels carry the gradient (through the geodesics, the redshift and
 * the emissivity); sky and horizon pixels are piecewise constant in p.
 * Recomputes trajectories from the checkpoints.  Synchronises `stream`. */
GG_API int gg_backward(gg_ctx* ctx, const double* dl_drgb_dev, double grad[5], void* stream);

/* ---- sky map ----------------------------------------------------------- */
/* Sets the context's equirectangular sky map, raytracer::curved::HdriSky
 * (crates/raytracer/src/curved/sky.rs:43-123): width*height linear RGB float
 * texels, row-major, row 0 = the +z pole, columns wrapping in azimuth
 * (decoding the .hdr file stays with the caller).  Copied to the device;
 * renders with opts.sky = GG_SKY_HDRI sample it bilinearly (wrap in x, clamp
 * in y) at the escape direction, scaled by `intensity`. */
GG_API int gg_set_hdri(gg_ctx* ctx, const float* rgb, uint32_t width, uint32_t height,
                       float intensity);

/* ---- scene of objects in the spatial slice ----------------------------- */
/* raytracer::shape::{Sphere, Quad} (crates/raytracer/src/shape/sphere.rs:9-87,
 * quad.rs:8-125) with the materials whose one-sample shading the curved
 * tracer's shade_hit (curved/tracer.rs:369-384) reads deterministically:
 * Lambertian (albedo), DiffuseLight (emission), Metal with fuzz 0 (albedo
 * when the mirror direction leaves the surface) and Dielectric (white).
 * Coordinates are the Cartesian image of Boyer-Lindquist (r, theta, phi):
 * (r sin th cos ph, r sin th sin ph, r cos th). */
#define GG_PRIM_SPHERE 0
#define GG_PRIM_QUAD 1
#define GG_MAT_LAMBERTIAN 0
#define GG_MAT_DIFFUSE_LIGHT 1
#define GG_MAT_METAL 2
#define GG_MAT_DIELECTRIC 3

typedef struct gg_prim_t {
  int32_t kind;      /* GG_PRIM_*                                          */
  int32_t material;  /* GG_MAT_*                                           */
  double p[3];       /* sphere centre, or quad corner Q                    */
  double u[3];       /* quad edge u                                        */
  double v[3];       /* quad edge v                                        */
  double radius;     /* sphere radius (> 0)                                */
  double color[3];   /* albedo (Lambertian, Metal) or emission (DiffuseLight) */
  double fuzz;       /* Metal: 0 (a fuzzed mirror samples a random direction) */
  double ior;        /* Dielectric index of refraction (shading ignores it) */
} gg_prim_t;

/* Sets the context's scene (copied; a bounding-volume hierarchy is built
 * over it).  n = 0 clears it.  Renders with opts.scene = 1 test each
 * accepted step's chord against it; rays whose chord hits end with
 * GG_CLASS_SCENE and the shaded, redshifted surface colour. */
GG_API int gg_set_scene(gg_ctx* ctx, const gg_prim_t* prims, uint32_t n);

/* The checks and hierarchy build of gg_set_scene without a device: GG_OK
 * (and, when not NULL, the hierarchy's node count and depth) or the error
 * gg_set_scene would return. */
GG_API int gg_scene_validate(const gg_prim_t* prims, uint32_t n, uint32_t* n_nodes,
                             uint32_t* depth);

/* ---- measurement ------------------------------------------------------- */
/* FMA throughput of the context's device in FLOP/s (an FMA counts 2), best
 * of 5 timed launches of independent FMA chains: fp64 = 1 for the FP64 pipe,
 * 0 for FP32.  The roofline denominator of the trace kernels.  No reference
 * counterpart (the reference has no device code). */
GG_API int gg_measure_fma_peak(gg_ctx* ctx, int fp64, double* flops);
/* sin and cos of n polar angles in FP32, by the routine the GG_PREC_MIXED
 * kernel's right-hand side uses (theta in [-pi/4, 5 pi/4]), evaluated on the
 * host from the same source so its accuracy can be checked without a GPU.
 * 0, or -1 for a NULL pointer.  No reference counterpart. */
GG_API int gg_polar_sincos(const float* theta, float* s, float* c, uint32_t n);

/* Device functions exported for bit-exact checks against the oracle on
 * identical inputs (test use; no reference counterpart).  Device pointers,
 * enqueued on `stream` (NULL = CUDA's default stream); 0, GG_ERR_INVALID_ARG
 * for a NULL pointer, GG_ERR_CUDA if the launch failed.
 * gg_check_procedural_sky: ProceduralSky::sample (sky.rs:26-40) of n unit
 *   directions dirs[3 i .. 3 i + 2] into rgb[3 i .. 3 i + 2].
 * gg_check_spatial_dir: spatial_dir (tracer.rs:185-189) of n velocities
 *   vel[4 i .. 4 i + 3] into dirs[3 i .. 3 i + 2]. */
GG_API int gg_check_procedural_sky(const double* dirs_dev, double* rgb_dev, uint64_t n,
                                   void* stream);
GG_API int gg_check_spatial_dir(const double* vel_dev, double* dirs_dev, uint64_t n,
                                void* stream);

/* Vector-Jacobian product of one Kerr right-hand side, the product the
 * differentiable render's backward takes at every stage (test use; no
 * reference counterpart).  in_dev: n points of 12 doubles (M, a, r, theta,
 * w[4], kb[4]); out_dev: n x 7 (kb . da/dr, da/dtheta, da/dw[0..3], da/da).
 * form 0: the hand-written reverse pass; 1: dual numbers.  Same pointer,
 * stream and return conventions as above; GG_ERR_INVALID_ARG for another form. */
GG_API int gg_check_kerr_vjp(const double* in_dev, double* out_dev, uint64_t n, int form,
                             void* stream);

/* The mixed form's step-size factor of an accepted attempt, (8 / s2)^(1/10)
 * for the squared error norm s2 (err = sqrt(s2 / 8) against tolerance 1;
 * s2 below 8e-60 taken as 8e-60), of n values (test use; no reference
 * counterpart; the reference's law is geodesic.rs:310-321).  Same pointer,
 * stream and return conventions as above. */
GG_API int gg_check_step_factor(const double* s2_dev, double* out_dev, uint64_t n, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* GARGANTUA_GPU_H */
