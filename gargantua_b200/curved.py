"""Host mirror of gargantua's ``raytracer::curved`` render API over the C ABI.

``render`` and ``render_with_disk`` keep the reference signatures
(crates/raytracer/src/curved/renderer.rs:82-101) and return the image as a
``uint8`` array of shape (height, width, 3), the ``RgbImage`` layout.  They
run the CUDA library; there is no CPU path.

``HdriSky`` is the reference's equirectangular environment map
(crates/raytracer/src/curved/sky.rs:43-123), sampled on the GPU.
``render_with_scene`` / ``render_with_disk_and_scene`` (renderer.rs:110-254)
test every step's chord against ``SceneObjects`` (spheres and quads) on the
GPU.

Extensions beyond the reference (all opt-in through ``RenderOptions`` or
``Scene``): a thin equatorial disk, a seeded checkerboard sky, seeded
jittered samples, a configurable step budget and integrator, the mixed
FP32/FP64 precision form, and per-sample outcome arrays.
"""
from __future__ import annotations

import ctypes as C
import itertools
import math
from dataclasses import dataclass, field
from typing import Optional, Union

import numpy as np

from . import abi
from .gr_core import Kerr, RK45Integrator, Schwarzschild, renderer_integrator

Metric = Union[Schwarzschild, Kerr]


@dataclass
class Camera:
    """Pinhole camera (crates/raytracer/src/curved/camera.rs:9-15)."""

    position: tuple = (0.0, 30.0, math.pi / 2.0, 0.0)
    look_at: tuple = (-1.0, 0.0, 0.0)
    up: tuple = (0.0, 0.0, 1.0)
    fov_y_radians: float = math.radians(60.0)
    aspect: float = 1.0

    @classmethod
    def inclined(cls, r: float, inclination: float, fov_y_radians: float,
                 aspect: float) -> "Camera":
        """Camera at (0, r, inclination, 0) looking at the hole with +z up."""
        c = abi.gg_camera_t()
        abi.check(abi.load().gg_camera_inclined(C.byref(c), r, inclination, fov_y_radians,
                                                aspect), "gg_camera_inclined")
        return cls(tuple(c.position), tuple(c.look_at), tuple(c.up), c.fov_y_radians, c.aspect)

    def to_c(self) -> abi.gg_camera_t:
        c = abi.gg_camera_t()
        c.position[:] = [float(x) for x in self.position]
        c.look_at[:] = [float(x) for x in self.look_at]
        c.up[:] = [float(x) for x in self.up]
        c.fov_y_radians = float(self.fov_y_radians)
        c.aspect = float(self.aspect)
        return c


@dataclass
class AccretionDisk:
    """Volumetric Gaussian disk (crates/raytracer/src/curved/disk.rs:8-31)."""

    r_inner: float = 6.0
    r_outer: float = 20.0
    scale_height: float = 1.0
    density_0: float = 1.0
    temperature_0: float = 1.0

    def to_c(self) -> abi.gg_disk_t:
        d = abi.gg_disk_t()
        d.kind = abi.GG_DISK_VOLUMETRIC
        d.r_inner, d.r_outer = self.r_inner, self.r_outer
        d.scale_height, d.density_0 = self.scale_height, self.density_0
        d.temperature_0 = self.temperature_0
        return d


@dataclass
class ThinDisk:
    """Thin equatorial disk: a ray ends at its first theta = pi/2 crossing with
    r in [r_inner, r_outer]; observed intensity g^4 (r_inner / r)^q and colour
    temperature g (r_inner / r)^(3/4), g the redshift of renderer's
    ``redshift_factor`` (tracer.rs:158-183)."""

    r_inner: float = 6.0
    r_outer: float = 20.0
    emissivity_index: float = 3.0

    def to_c(self) -> abi.gg_disk_t:
        d = abi.gg_disk_t()
        d.kind = abi.GG_DISK_THIN
        d.r_inner, d.r_outer = self.r_inner, self.r_outer
        d.emissivity_index = self.emissivity_index
        d.temperature_0 = 1.0
        return d


@dataclass
class ProceduralSky:
    """The reference's hashed starfield (crates/raytracer/src/curved/sky.rs:19-41)."""


@dataclass
class CheckerSky:
    """Seeded checkerboard over the escape point's (theta, phi)."""

    rows: int = 18
    cols: int = 36
    seed: int = 0


# Serial numbers of sky maps and scenes, by which a Renderer knows what it
# has uploaded.
_SERIALS = itertools.count(1)


class HdriSky:
    """Equirectangular environment map (sky.rs:43-123): linear RGB float32
    texels, shape (height, width, 3), row 0 at the +z pole, columns wrapping
    in azimuth; bilinear with wrap in x and clamp in y, times ``intensity``.

    A Renderer uploads the map the first time a render meets this object
    (and again after ``with_intensity`` or ``set_pixels``)."""

    def __init__(self, pixels, intensity: float = 1.0):
        self.set_pixels(pixels)
        self.intensity = float(intensity)

    @classmethod
    def from_pixels(cls, width: int, height: int, pixels) -> "HdriSky":
        """HdriSky::from_pixels (sky.rs:75-78): width*height RGB triples, row-major."""
        px = np.asarray(pixels, np.float32)
        if px.size != width * height * 3:
            raise ValueError("pixel buffer size mismatch")
        return cls(px.reshape(height, width, 3))

    @classmethod
    def from_file(cls, path) -> "HdriSky":
        """HdriSky::from_file (sky.rs:59-71) for Radiance .hdr files."""
        from .hdr import read_hdr
        return cls(read_hdr(path))

    def with_intensity(self, intensity: float) -> "HdriSky":
        self.intensity = float(intensity)
        return self

    def set_pixels(self, pixels) -> None:
        px = np.ascontiguousarray(pixels, np.float32)
        if px.ndim != 3 or px.shape[2] != 3 or px.shape[0] < 1 or px.shape[1] < 1:
            raise ValueError("HdriSky pixels must be (height, width, 3)")
        self.pixels = px
        self.version = getattr(self, "version", 0) + 1
        if not hasattr(self, "_serial"):
            self._serial = next(_SERIALS)

    @property
    def width(self) -> int:
        return self.pixels.shape[1]

    @property
    def height(self) -> int:
        return self.pixels.shape[0]

    def key(self):
        # a serial number, not id(): a new object may reuse a freed one's id
        return (self._serial, self.version, self.intensity)


@dataclass
class Lambertian:
    """crates/raytracer/src/material/lambertian.rs: shaded with its albedo."""
    albedo: tuple = (0.5, 0.5, 0.5)
    kind = abi.GG_MAT_LAMBERTIAN

    def color(self):
        return self.albedo


@dataclass
class DiffuseLight:
    """material/diffuse_light.rs: emits, does not scatter."""
    emit: tuple = (1.0, 1.0, 1.0)
    kind = abi.GG_MAT_DIFFUSE_LIGHT

    def color(self):
        return self.emit


@dataclass
class Metal:
    """material/metal.rs; only fuzz = 0 renders (a fuzzed mirror's one-sample
    shading depends on a random direction)."""
    albedo: tuple = (0.8, 0.8, 0.8)
    fuzz: float = 0.0
    kind = abi.GG_MAT_METAL

    def color(self):
        return self.albedo


@dataclass
class Dielectric:
    """material/dielectric.rs: always scatters, with white attenuation."""
    ior: float = 1.5
    kind = abi.GG_MAT_DIELECTRIC

    def color(self):
        return (1.0, 1.0, 1.0)


@dataclass
class Sphere:
    """crates/raytracer/src/shape/sphere.rs:9-87."""
    center: tuple
    radius: float
    material: object


@dataclass
class Quad:
    """Parallelogram Q + a u + b v, a, b in [0, 1] (shape/quad.rs:8-125)."""
    q: tuple
    u: tuple
    v: tuple
    material: object


class SceneObjects:
    """A list of objects for the curved tracer, like ``World`` (scene/world.rs)
    with ``add`` chaining; a Renderer uploads it (gg_set_scene, which builds
    the bounding-volume hierarchy) the first time a render meets it, and
    again after ``add``."""

    def __init__(self, objects=()):
        self.objects = []
        self.version = 0
        self._serial = next(_SERIALS)
        for o in objects:
            self.add(o)

    def add(self, obj) -> "SceneObjects":
        if not isinstance(obj, (Sphere, Quad)):
            raise TypeError("scene objects are Sphere or Quad")
        self.objects.append(obj)
        self.version += 1
        return self

    def __len__(self) -> int:
        return len(self.objects)

    def key(self):
        return (self._serial, self.version)

    def to_c(self):
        arr = (abi.gg_prim_t * len(self.objects))()
        for k, o in enumerate(self.objects):
            p = arr[k]
            m = o.material
            p.material = m.kind
            p.color[:] = [float(x) for x in m.color()]
            p.fuzz = float(getattr(m, "fuzz", 0.0))
            p.ior = float(getattr(m, "ior", 0.0))
            if isinstance(o, Sphere):
                p.kind = abi.GG_PRIM_SPHERE
                p.p[:] = [float(x) for x in o.center]
                p.radius = float(o.radius)
            else:
                p.kind = abi.GG_PRIM_QUAD
                p.p[:] = [float(x) for x in o.q]
                p.u[:] = [float(x) for x in o.u]
                p.v[:] = [float(x) for x in o.v]
        return arr


@dataclass
class RenderOptions:
    """``RenderOptions`` (renderer.rs:17-26) plus the extensions listed above."""

    samples_per_axis: int = 1
    show_progress: bool = False
    sky: Union[ProceduralSky, CheckerSky, HdriSky, None] = None
    jitter_spp: int = 0
    seed: int = 0
    max_steps: int = 5000
    integrator: Optional[RK45Integrator] = None
    precision: int = abi.GG_PREC_FP64
    attempt_budget: int = 0
    row_offset: int = 0   # with row_step > 1: trace rows row_offset, row_offset + row_step, ...
    row_step: int = 1

    def to_c(self) -> abi.gg_render_opts_t:
        o = abi.gg_render_opts_t()
        o.samples_per_axis = max(1, int(self.samples_per_axis))
        o.jitter_spp = int(self.jitter_spp)
        o.seed = int(self.seed) & (2**64 - 1)
        sky = self.sky or ProceduralSky()
        if isinstance(sky, CheckerSky):
            o.sky, o.sky_rows, o.sky_cols = abi.GG_SKY_CHECKER, sky.rows, sky.cols
            o.sky_seed = int(sky.seed) & (2**64 - 1)
        elif isinstance(sky, HdriSky):
            o.sky, o.sky_rows, o.sky_cols, o.sky_seed = abi.GG_SKY_HDRI, 18, 36, 0
        else:
            o.sky, o.sky_rows, o.sky_cols, o.sky_seed = abi.GG_SKY_PROCEDURAL, 18, 36, 0
        o.attempt_budget = int(self.attempt_budget)
        o.row_offset = int(self.row_offset)
        o.row_step = max(1, int(self.row_step))
        return o


@dataclass
class Scene:
    """Everything one render call needs, as the C ABI takes it."""

    metric: Metric
    camera: Camera
    width: int
    height: int
    disk: Union[AccretionDisk, ThinDisk, None] = None
    options: RenderOptions = field(default_factory=RenderOptions)
    objects: Optional[SceneObjects] = None  # render_with_scene: chords against these

    @property
    def spp(self) -> int:
        o = self.options
        return o.jitter_spp if o.jitter_spp > 0 else max(1, o.samples_per_axis) ** 2

    @property
    def n_samples(self) -> int:
        return self.width * self.rows * self.spp

    @property
    def rows(self) -> int:
        """Image rows this render traces (all of them unless the options
        select every row_step-th row from row_offset)."""
        step = max(1, int(self.options.row_step))
        off = int(self.options.row_offset)
        return 0 if off >= self.height else (self.height - off + step - 1) // step

    def integrator_c(self) -> abi.gg_integrator_t:
        integ = self.options.integrator or renderer_integrator()
        return integ.to_c(self.options.max_steps, self.options.precision)

    def c_structs(self):
        o = self.options.to_c()
        o.scene = 1 if self.objects is not None else 0
        return (self.metric.to_c(), self.camera.to_c(),
                self.disk.to_c() if self.disk is not None else None, self.integrator_c(), o)

    def c_args(self):
        m, c, d, i, o = self.c_structs()
        self._keep = (m, c, d, i, o)
        return (C.byref(m), C.byref(c), C.byref(d) if d is not None else None, C.byref(i),
                C.byref(o), C.c_uint32(self.width), C.c_uint32(self.height))


class RayOutputs:
    """Host arrays of per-sample outcomes (``gg_ray_out_t``)."""

    def __init__(self, n: int):
        self.n = n
        self.cls = np.full(n, -1, np.int32)
        self.x = np.zeros((4, n), np.float64)
        self.v = np.zeros((4, n), np.float64)
        self.lam = np.zeros(n, np.float64)
        self.attempts = np.zeros(n, np.uint32)
        self.accepted = np.zeros(n, np.uint32)
        self.intensity = np.zeros(n, np.float64)
        self.color_temp = np.zeros(n, np.float64)
        self.rgb = np.zeros((n, 3), np.float64)
        self.cross = np.zeros((8, n), np.float64)

    def struct(self) -> abi.gg_ray_out_t:
        def p(a, t):
            return a.ctypes.data_as(C.POINTER(t))
        return abi.gg_ray_out_t(p(self.cls, C.c_int32), p(self.x, C.c_double),
                                p(self.v, C.c_double), p(self.lam, C.c_double),
                                p(self.attempts, C.c_uint32), p(self.accepted, C.c_uint32),
                                p(self.intensity, C.c_double), p(self.color_temp, C.c_double),
                                p(self.rgb, C.c_double), p(self.cross, C.c_double))


class Renderer:
    """One library context (one CUDA stream) on one device."""

    def __init__(self, device: int = 0):
        self._lib = abi.load()
        h = C.c_void_p()
        abi.check(self._lib.gg_create(C.byref(h), int(device)), "gg_create")
        self._h = h
        self._hdri_key = None
        self._scene_key = None

    def close(self) -> None:
        if self._h:
            self._lib.gg_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    @property
    def stream(self) -> int:
        return self._lib.gg_stream(self._h) or 0

    def set_hdri(self, sky: HdriSky) -> None:
        """Uploads `sky`'s map to this context (gg_set_hdri)."""
        px = sky.pixels
        abi.check(self._lib.gg_set_hdri(self._h, px.ctypes.data_as(C.c_void_p), px.shape[1],
                                        px.shape[0], C.c_float(sky.intensity)), "gg_set_hdri")
        self._hdri_key = sky.key()

    def set_scene(self, objects: SceneObjects) -> None:
        """Uploads `objects` to this context (gg_set_scene)."""
        arr = objects.to_c()
        abi.check(self._lib.gg_set_scene(self._h, arr, len(arr)), "gg_set_scene")
        self._scene_key = objects.key()

    def _sky_map(self, scene: Scene) -> None:
        sky = scene.options.sky
        if isinstance(sky, HdriSky) and sky.key() != self._hdri_key:
            self.set_hdri(sky)
        if scene.objects is not None and scene.objects.key() != self._scene_key:
            self.set_scene(scene.objects)

    def render(self, scene: Scene, rays: bool = False):
        """Synchronous render into host memory: (image, RayOutputs or None)."""
        img = np.zeros((scene.rows, scene.width, 3), np.uint8)
        out = RayOutputs(scene.n_samples) if rays else None
        self._sky_map(scene)
        st = self._lib.gg_render(self._h, *scene.c_args(), img.ctypes.data_as(C.c_void_p),
                                 C.byref(out.struct()) if out else None)
        abi.check(st, "gg_render")
        return img, out

    def render_into(self, scene: Scene, rgb_host: np.ndarray) -> None:
        """Synchronous render into a caller-owned (e.g. pinned) uint8 host buffer."""
        assert rgb_host.dtype == np.uint8 and rgb_host.size >= scene.width * scene.rows * 3
        self._sky_map(scene)
        st = self._lib.gg_render(self._h, *scene.c_args(), rgb_host.ctypes.data_as(C.c_void_p),
                                 None)
        abi.check(st, "gg_render")

    def fma_peak(self, fp64: bool = True) -> float:
        """Measured FMA throughput of this device in FLOP/s."""
        f = C.c_double()
        abi.check(self._lib.gg_measure_fma_peak(self._h, 1 if fp64 else 0, C.byref(f)),
                  "gg_measure_fma_peak")
        return f.value

    def render_device(self, scene: Scene, rgb_dev: int, rays_dev: abi.gg_ray_out_t | None = None,
                      stream: int | None = None) -> None:
        """Enqueue a render writing device pointers (no synchronisation).

        ``stream`` is a cudaStream_t handle; None or 0 is CUDA's default stream."""
        self._sky_map(scene)
        st = self._lib.gg_render_device(self._h, *scene.c_args(), C.c_void_p(rgb_dev),
                                        C.byref(rays_dev) if rays_dev is not None else None,
                                        C.c_void_p(stream or 0))
        abi.check(st, "gg_render_device")

    # ---- batches ------------------------------------------------------------
    @staticmethod
    def _batch_structs(scenes):
        """gg_scene_t array of `scenes`, and the batch's integrator and options
        (the first scene's: every scene of a batch shares them)."""
        arr = (abi.gg_scene_t * len(scenes))()
        keep = []
        for k, sc in enumerate(scenes):
            m, c, d, _, o = sc.c_structs()
            arr[k].metric = m
            arr[k].camera = c
            if d is not None:
                arr[k].disk = d
            arr[k].width = sc.width
            arr[k].height = sc.height
            arr[k].sky_seed = o.sky_seed
            keep.append((m, c, d, o))
        _, _, _, integ, opts = scenes[0].c_structs()
        return arr, integ, opts, keep

    def render_batch(self, scenes) -> list:
        """Synchronous batched render (gg_render_batch): one image per scene."""
        arr, integ, opts, _ = self._batch_structs(scenes)
        imgs = [np.zeros((sc.height, sc.width, 3), np.uint8) for sc in scenes]
        ptrs = (C.c_void_p * len(scenes))(*[im.ctypes.data for im in imgs])
        abi.check(self._lib.gg_render_batch(self._h, arr, len(scenes), C.byref(integ),
                                            C.byref(opts), ptrs), "gg_render_batch")
        return imgs

    def render_batch_device(self, scenes, rgb_dev: int, stream: int | None = None) -> None:
        """Enqueue a batched render writing the concatenated images to rgb_dev."""
        arr, integ, opts, _ = self._batch_structs(scenes)
        abi.check(self._lib.gg_render_batch_device(self._h, arr, len(scenes), C.byref(integ),
                                                   C.byref(opts), C.c_void_p(rgb_dev),
                                                   C.c_void_p(stream or 0)),
                  "gg_render_batch_device")

    def batch_autotune(self, scenes):
        """Times the batch kernel variants on `scenes`, keeps the fastest for
        this context; returns (variant, per-variant ms)."""
        arr, integ, opts, _ = self._batch_structs(scenes)
        v = C.c_int(-1)
        ms = (C.c_double * abi.GG_BATCH_VARIANTS)()
        abi.check(self._lib.gg_batch_autotune(self._h, arr, len(scenes), C.byref(integ),
                                              C.byref(opts), C.byref(v), ms),
                  "gg_batch_autotune")
        return v.value, list(ms)

    def batch_set_variant(self, variant: int) -> None:
        abi.check(self._lib.gg_batch_set_variant(self._h, int(variant)), "gg_batch_set_variant")

    def stats(self) -> abi.gg_stats_t:
        s = abi.gg_stats_t()
        abi.check(self._lib.gg_last_stats(self._h, C.byref(s)), "gg_last_stats")
        return s


_DEFAULT: Optional[Renderer] = None


def _renderer() -> Renderer:
    global _DEFAULT
    if _DEFAULT is None:
        _DEFAULT = Renderer(0)
    return _DEFAULT


def render(metric: Metric, camera: Camera, width: int, height: int,
           opts: Optional[RenderOptions] = None) -> np.ndarray:
    """``render`` (renderer.rs:82-90): sky / horizon only."""
    scene = Scene(metric, camera, width, height, None, opts or RenderOptions())
    return _renderer().render(scene)[0]


def render_with_disk(metric: Metric, camera: Camera, disk: Union[AccretionDisk, ThinDisk],
                     width: int, height: int, opts: Optional[RenderOptions] = None) -> np.ndarray:
    """``render_with_disk`` (renderer.rs:92-101)."""
    scene = Scene(metric, camera, width, height, disk, opts or RenderOptions())
    return _renderer().render(scene)[0]


def render_with_scene(metric: Metric, camera: Camera, objects: SceneObjects, width: int,
                      height: int, opts: Optional[RenderOptions] = None) -> np.ndarray:
    """``render_with_scene`` (renderer.rs:110-182)."""
    scene = Scene(metric, camera, width, height, None, opts or RenderOptions(), objects)
    return _renderer().render(scene)[0]


def render_with_disk_and_scene(metric: Metric, camera: Camera, disk: AccretionDisk,
                               objects: SceneObjects, width: int, height: int,
                               opts: Optional[RenderOptions] = None) -> np.ndarray:
    """``render_with_disk_and_scene`` (renderer.rs:184-254)."""
    scene = Scene(metric, camera, width, height, disk, opts or RenderOptions(), objects)
    return _renderer().render(scene)[0]


__all__ = ["Camera", "AccretionDisk", "ThinDisk", "ProceduralSky", "CheckerSky", "HdriSky",
           "Lambertian", "DiffuseLight", "Metal", "Dielectric", "Sphere", "Quad",
           "SceneObjects", "RenderOptions", "Scene", "RayOutputs", "Renderer", "render",
           "render_with_disk", "render_with_scene", "render_with_disk_and_scene"]
