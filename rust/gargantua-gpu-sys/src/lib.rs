//! Raw declarations of `include/gargantua_gpu.h`: the B200 ray path's C ABI.
//!
//! Every struct is `#[repr(C)]` with the header's fields in the header's
//! order; every entry point returns the header's status codes (0 = OK,
//! negative = `GG_ERR_*`, text through `gg_strerror`).  Nothing here
//! allocates or panics; the safe wrapper is the `gargantua-gpu` crate.
#![allow(non_camel_case_types)]

use std::os::raw::{c_char, c_int, c_void};

// ---- status ---------------------------------------------------------------
pub const GG_OK: c_int = 0;
pub const GG_ERR_INVALID_ARG: c_int = -1;
pub const GG_ERR_CUDA: c_int = -2;
pub const GG_ERR_OOM: c_int = -3;
pub const GG_ERR_BUDGET: c_int = -4;
pub const GG_ERR_UNSUPPORTED: c_int = -5;
pub const GG_ERR_NO_DEVICE: c_int = -6;
pub const GG_ERR_TOO_LARGE: c_int = -7;

// ---- enumerations ---------------------------------------------------------
pub const GG_METRIC_SCHWARZSCHILD: i32 = 0;
pub const GG_METRIC_KERR: i32 = 1;
pub const GG_DISK_NONE: i32 = 0;
pub const GG_DISK_VOLUMETRIC: i32 = 1;
pub const GG_DISK_THIN: i32 = 2;
pub const GG_PREC_FP64: i32 = 0;
pub const GG_PREC_MIXED: i32 = 1;
pub const GG_STEPPER_REFERENCE: i32 = 0;
pub const GG_STEPPER_DP45: i32 = 1;
pub const GG_SKY_PROCEDURAL: i32 = 0;
pub const GG_SKY_CHECKER: i32 = 1;
pub const GG_SKY_HDRI: i32 = 2;
pub const GG_CLASS_HORIZON: i32 = 0;
pub const GG_CLASS_ESCAPED: i32 = 1;
pub const GG_CLASS_DISK: i32 = 2;
pub const GG_CLASS_MAXSTEPS: i32 = 3;
pub const GG_CLASS_BUDGET: i32 = 4;
pub const GG_CLASS_SCENE: i32 = 5;
pub const GG_N_CLASSES: usize = 6;
pub const GG_BATCH_VARIANTS: usize = 12;
pub const GG_PRIM_SPHERE: i32 = 0;
pub const GG_PRIM_QUAD: i32 = 1;
pub const GG_MAT_LAMBERTIAN: i32 = 0;
pub const GG_MAT_DIFFUSE_LIGHT: i32 = 1;
pub const GG_MAT_METAL: i32 = 2;
pub const GG_MAT_DIELECTRIC: i32 = 3;

// ---- parameter structs ----------------------------------------------------
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct gg_metric_t {
    pub kind: i32,
    pub reserved: i32,
    pub mass: f64,
    pub spin: f64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct gg_camera_t {
    pub position: [f64; 4],
    pub look_at: [f64; 3],
    pub up: [f64; 3],
    pub fov_y_radians: f64,
    pub aspect: f64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct gg_disk_t {
    pub kind: i32,
    pub reserved: i32,
    pub r_inner: f64,
    pub r_outer: f64,
    pub scale_height: f64,
    pub density_0: f64,
    pub temperature_0: f64,
    pub emissivity_index: f64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct gg_integrator_t {
    pub initial_step: f64,
    pub min_step: f64,
    pub max_step: f64,
    pub tolerance: f64,
    pub max_radius: f64,
    pub horizon_buffer: f64,
    pub rtol: f64,
    pub atol: f64,
    pub max_steps: u32,
    pub precision: i32,
    pub stepper: i32,
    pub reserved: i32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct gg_render_opts_t {
    pub samples_per_axis: u32,
    pub jitter_spp: u32,
    pub seed: u64,
    pub sky: i32,
    pub sky_rows: u32,
    pub sky_cols: u32,
    pub row_offset: u32,
    pub sky_seed: u64,
    pub attempt_budget: u64,
    pub row_step: u32,
    pub scene: u32,
}

/// Per-sample outputs, each a nullable pointer (host memory for `gg_render`,
/// device memory for `gg_render_device`).
#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct gg_ray_out_t {
    pub cls: *mut i32,
    pub x: *mut f64,
    pub v: *mut f64,
    pub lambda: *mut f64,
    pub attempts: *mut u32,
    pub accepted: *mut u32,
    pub intensity: *mut f64,
    pub color_temp: *mut f64,
    pub rgb: *mut f64,
    pub cross: *mut f64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct gg_stats_t {
    pub rays: u64,
    pub attempts: u64,
    pub accepted: u64,
    pub class_count: [u64; GG_N_CLASSES],
    pub kernel_ms: f64,
    pub fp64_rays: u64,
    pub fp64_attempts: u64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct gg_scene_t {
    pub metric: gg_metric_t,
    pub camera: gg_camera_t,
    pub disk: gg_disk_t,
    pub width: u32,
    pub height: u32,
    pub sky_seed: u64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct gg_prim_t {
    pub kind: i32,
    pub material: i32,
    pub p: [f64; 3],
    pub u: [f64; 3],
    pub v: [f64; 3],
    pub radius: f64,
    pub color: [f64; 3],
    pub fuzz: f64,
    pub ior: f64,
}

/// Opaque library context (one CUDA stream and its device scratch).
#[repr(C)]
pub struct gg_ctx {
    _private: [u8; 0],
}

// ---- entry points ---------------------------------------------------------
extern "C" {
    pub fn gg_version() -> *const c_char;
    pub fn gg_strerror(status: c_int) -> *const c_char;
    pub fn gg_struct_size(name: *const c_char) -> c_int;

    pub fn gg_metric_schwarzschild(out: *mut gg_metric_t, mass: f64) -> c_int;
    pub fn gg_metric_kerr(out: *mut gg_metric_t, mass: f64, spin: f64) -> c_int;
    pub fn gg_integrator_default(out: *mut gg_integrator_t);
    pub fn gg_disk_default(out: *mut gg_disk_t);
    pub fn gg_render_opts_default(out: *mut gg_render_opts_t);
    pub fn gg_camera_inclined(out: *mut gg_camera_t, r: f64, inclination_rad: f64,
                              fov_y_radians: f64, aspect: f64) -> c_int;
    pub fn gg_kerr_isco(mass: f64, spin: f64) -> f64;
    pub fn gg_kerr_photon_orbit(mass: f64, spin: f64) -> f64;
    pub fn gg_validate(metric: *const gg_metric_t, camera: *const gg_camera_t,
                       disk: *const gg_disk_t, integ: *const gg_integrator_t,
                       opts: *const gg_render_opts_t, width: u32, height: u32) -> c_int;

    pub fn gg_create(out: *mut *mut gg_ctx, device: c_int) -> c_int;
    pub fn gg_destroy(ctx: *mut gg_ctx) -> c_int;
    pub fn gg_stream(ctx: *mut gg_ctx) -> *mut c_void;
    pub fn gg_last_stats(ctx: *mut gg_ctx, out: *mut gg_stats_t) -> c_int;

    pub fn gg_render(ctx: *mut gg_ctx, metric: *const gg_metric_t, camera: *const gg_camera_t,
                     disk: *const gg_disk_t, integ: *const gg_integrator_t,
                     opts: *const gg_render_opts_t, width: u32, height: u32, rgb_out: *mut u8,
                     rays_out: *const gg_ray_out_t) -> c_int;
    pub fn gg_render_device(ctx: *mut gg_ctx, metric: *const gg_metric_t,
                            camera: *const gg_camera_t, disk: *const gg_disk_t,
                            integ: *const gg_integrator_t, opts: *const gg_render_opts_t,
                            width: u32, height: u32, rgb_dev: *mut u8,
                            rays_dev: *const gg_ray_out_t, stream: *mut c_void) -> c_int;
    pub fn gg_render_device_noalloc(metric: *const gg_metric_t, camera: *const gg_camera_t,
                                    disk: *const gg_disk_t, integ: *const gg_integrator_t,
                                    opts: *const gg_render_opts_t, width: u32, height: u32,
                                    rgb_dev: *mut u8, rays_dev: *const gg_ray_out_t,
                                    stream: *mut c_void) -> c_int;

    pub fn gg_render_batch_device(ctx: *mut gg_ctx, scenes: *const gg_scene_t, n: u32,
                                  integ: *const gg_integrator_t, opts: *const gg_render_opts_t,
                                  rgb_dev: *mut u8, stream: *mut c_void) -> c_int;
    pub fn gg_render_batch(ctx: *mut gg_ctx, scenes: *const gg_scene_t, n: u32,
                           integ: *const gg_integrator_t, opts: *const gg_render_opts_t,
                           rgb_out: *const *mut u8) -> c_int;
    pub fn gg_batch_autotune(ctx: *mut gg_ctx, scenes: *const gg_scene_t, n: u32,
                             integ: *const gg_integrator_t, opts: *const gg_render_opts_t,
                             variant_out: *mut c_int, ms_out: *mut f64) -> c_int;
    pub fn gg_batch_set_variant(ctx: *mut gg_ctx, variant: c_int) -> c_int;
    pub fn gg_batch_variant_info(v: c_int, out: *mut i32) -> c_int;

    pub fn gg_forward_ckpt(ctx: *mut gg_ctx, metric: *const gg_metric_t, r_cam: f64,
                           inclination: f64, fov_y_radians: f64, aspect: f64,
                           disk: *const gg_disk_t, integ: *const gg_integrator_t,
                           opts: *const gg_render_opts_t, width: u32, height: u32,
                           rgb_lin_dev: *mut f64, stream: *mut c_void) -> c_int;
    pub fn gg_backward(ctx: *mut gg_ctx, dl_drgb_dev: *const f64, grad: *mut f64,
                       stream: *mut c_void) -> c_int;

    pub fn gg_set_hdri(ctx: *mut gg_ctx, rgb: *const f32, width: u32, height: u32,
                       intensity: f32) -> c_int;
    pub fn gg_set_scene(ctx: *mut gg_ctx, prims: *const gg_prim_t, n: u32) -> c_int;
    pub fn gg_scene_validate(prims: *const gg_prim_t, n: u32, n_nodes: *mut u32,
                             depth: *mut u32) -> c_int;

    pub fn gg_measure_fma_peak(ctx: *mut gg_ctx, fp64: c_int, flops: *mut f64) -> c_int;
    pub fn gg_polar_sincos(theta: *const f32, s: *mut f32, c: *mut f32, n: u32) -> c_int;
    pub fn gg_check_procedural_sky(dirs_dev: *const f64, rgb_dev: *mut f64, n: u64,
                                   stream: *mut c_void) -> c_int;
    pub fn gg_check_spatial_dir(vel_dev: *const f64, dirs_dev: *mut f64, n: u64,
                                stream: *mut c_void) -> c_int;
    pub fn gg_check_kerr_vjp(in_dev: *const f64, out_dev: *mut f64, n: u64, form: c_int,
                             stream: *mut c_void) -> c_int;
    pub fn gg_check_step_factor(s2_dev: *const f64, out_dev: *mut f64, n: u64,
                                stream: *mut c_void) -> c_int;
}
