//! The B200 ray path behind gargantua's own render calls.
//!
//! `render` and `render_with_disk` keep the signatures of
//! `raytracer::curved::render` / `render_with_disk` (renderer.rs:82-101) and
//! panic with the library's message where the CPU renderer cannot fail;
//! `try_render` / `try_render_with_disk` return the error instead.  The metric
//! generic is the small `GpuMetric` trait, implemented for gr-core's
//! `Schwarzschild` and `Kerr`.  One library context (one CUDA stream) per
//! host thread.

use gargantua_gpu_sys as sys;
use gr_core::{Kerr, Schwarzschild};
use image::RgbImage;
use raytracer::curved::renderer::RenderOptions;
use raytracer::curved::{AccretionDisk, Camera};
use std::ffi::CStr;

/// A status from the library (`GG_ERR_*`) with its text.
#[derive(Debug, thiserror::Error)]
#[error("gargantua-gpu: {message} (status {status})")]
pub struct GpuError {
    pub status: i32,
    pub message: String,
}

fn check(status: i32) -> Result<(), GpuError> {
    if status == sys::GG_OK {
        return Ok(());
    }
    let message = unsafe { CStr::from_ptr(sys::gg_strerror(status)) }
        .to_string_lossy()
        .into_owned();
    Err(GpuError { status, message })
}

/// A metric the GPU path traces: its POD form.
pub trait GpuMetric {
    fn to_gg(&self) -> sys::gg_metric_t;
}

impl GpuMetric for Schwarzschild {
    fn to_gg(&self) -> sys::gg_metric_t {
        sys::gg_metric_t { kind: sys::GG_METRIC_SCHWARZSCHILD, reserved: 0, mass: self.mass,
                           spin: 0.0 }
    }
}

impl GpuMetric for Kerr {
    // Kerr::new has already asserted the mass and clamped the spin (kerr.rs:29-34)
    fn to_gg(&self) -> sys::gg_metric_t {
        sys::gg_metric_t { kind: sys::GG_METRIC_KERR, reserved: 0, mass: self.mass,
                           spin: self.spin }
    }
}

struct Ctx(*mut sys::gg_ctx);

impl Drop for Ctx {
    fn drop(&mut self) {
        if !self.0.is_null() {
            unsafe { sys::gg_destroy(self.0) };
        }
    }
}

thread_local! {
    static CTX: std::cell::RefCell<Option<Ctx>> = const { std::cell::RefCell::new(None) };
}

fn with_ctx<T>(f: impl FnOnce(*mut sys::gg_ctx) -> Result<T, GpuError>) -> Result<T, GpuError> {
    CTX.with(|cell| {
        let mut slot = cell.borrow_mut();
        if slot.is_none() {
            let mut c = std::ptr::null_mut();
            check(unsafe { sys::gg_create(&mut c, 0) })?;
            *slot = Some(Ctx(c));
        }
        f(slot.as_ref().unwrap().0)
    })
}

fn camera_pod(camera: &Camera) -> sys::gg_camera_t {
    sys::gg_camera_t {
        position: [camera.position[0], camera.position[1], camera.position[2],
                   camera.position[3]],
        look_at: [camera.look_at.x, camera.look_at.y, camera.look_at.z],
        up: [camera.up.x, camera.up.y, camera.up.z],
        fov_y_radians: camera.fov_y_radians,
        aspect: camera.aspect,
    }
}

fn render_inner<M: GpuMetric>(metric: &M, camera: &Camera, disk: Option<&AccretionDisk>,
                              width: u32, height: u32, opts: &RenderOptions)
                              -> Result<RgbImage, GpuError> {
    let m = metric.to_gg();
    let cam = camera_pod(camera);
    // the integrator render_inner builds (renderer.rs:264-265): r_max = 200,
    // 5,000 step() calls
    let mut integ = sys::gg_integrator_t::default();
    unsafe { sys::gg_integrator_default(&mut integ) };
    let mut o = sys::gg_render_opts_t::default();
    unsafe { sys::gg_render_opts_default(&mut o) };
    o.samples_per_axis = opts.samples_per_axis.max(1);
    let d = disk.map(|d| sys::gg_disk_t {
        kind: sys::GG_DISK_VOLUMETRIC,
        reserved: 0,
        r_inner: d.r_inner,
        r_outer: d.r_outer,
        scale_height: d.scale_height,
        density_0: d.density_0,
        temperature_0: d.temperature_0,
        emissivity_index: 3.0,
    });
    let disk_ptr = d.as_ref().map_or(std::ptr::null(), |d| d as *const sys::gg_disk_t);
    let mut img = RgbImage::new(width, height); // row-major RGB8, the layout gg_render writes
    with_ctx(|ctx| {
        check(unsafe {
            sys::gg_render(ctx, &m, &cam, disk_ptr, &integ, &o, width, height,
                           img.as_mut_ptr(), std::ptr::null())
        })
    })?;
    Ok(img)
}

/// `raytracer::curved::render` on the GPU, or the library's error.
pub fn try_render<M: GpuMetric>(metric: &M, camera: &Camera, width: u32, height: u32,
                                opts: RenderOptions) -> Result<RgbImage, GpuError> {
    render_inner(metric, camera, None, width, height, &opts)
}

/// `raytracer::curved::render_with_disk` on the GPU, or the library's error.
pub fn try_render_with_disk<M: GpuMetric>(metric: &M, camera: &Camera, disk: &AccretionDisk,
                                          width: u32, height: u32, opts: RenderOptions)
                                          -> Result<RgbImage, GpuError> {
    render_inner(metric, camera, Some(disk), width, height, &opts)
}

/// Drop-in for `raytracer::curved::render` (renderer.rs:82-90).
pub fn render<M: GpuMetric>(metric: &M, camera: &Camera, width: u32, height: u32,
                            opts: RenderOptions) -> RgbImage {
    try_render(metric, camera, width, height, opts).unwrap_or_else(|e| panic!("{e}"))
}

/// Drop-in for `raytracer::curved::render_with_disk` (renderer.rs:92-101).
pub fn render_with_disk<M: GpuMetric>(metric: &M, camera: &Camera, disk: &AccretionDisk,
                                      width: u32, height: u32, opts: RenderOptions)
                                      -> RgbImage {
    try_render_with_disk(metric, camera, disk, width, height, opts)
        .unwrap_or_else(|e| panic!("{e}"))
}
