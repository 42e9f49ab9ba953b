"""Python loader of the CPU oracle (``oracle/_build/liboracle_gg.so``).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke`` and the
CPU-baseline leg of ``bench.py`` as the checker; the product never imports it.
The parameter structs are the product ABI's POD structs so both sides trace
identical inputs.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

from gargantua_b200 import abi

ORACLE_DIR = Path(__file__).resolve().parent
LIB_PATH = ORACLE_DIR / "_build" / "liboracle_gg.so"

P = C.POINTER
D4 = C.c_double * 4


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(ORACLE_DIR)], check=True)
    return LIB_PATH


VARIANT_PATHS = {
    "plain": LIB_PATH,
    # same algorithm rounded differently; used only to measure each ray's
    # sensitivity to last-bit rounding, never as the reference
    "fma": ORACLE_DIR / "_build" / "liboracle_gg_fma.so",
    "alt": ORACLE_DIR / "_build" / "liboracle_gg_alt.so",
}
_LIBS: dict = {}


def lib(variant: str = "plain") -> C.CDLL:
    """The oracle library, or one of its rounding-perturbed builds."""
    path = VARIANT_PATHS[variant]
    if path not in _LIBS:
        if not path.exists():
            build()
        L = C.CDLL(str(path))
        common = [P(abi.gg_metric_t), P(abi.gg_camera_t), P(abi.gg_disk_t),
                  P(abi.gg_integrator_t), P(abi.gg_render_opts_t), C.c_uint32, C.c_uint32]
        sig = {
            "ggo_render": (C.c_int, common + [C.c_void_p, P(abi.gg_ray_out_t), C.c_int]),
            "ggo_trace_samples": (C.c_int, common + [C.c_void_p, C.c_uint64,
                                                     P(abi.gg_ray_out_t), C.c_int]),
            "ggo_trace_cross": (C.c_int, common + [C.c_void_p, C.c_uint64, C.c_void_p,
                                                   C.c_int]),
            "ggo_trace_state": (C.c_int, common[:5] + [C.c_void_p, P(abi.gg_ray_out_t)]),
            "ggo_trace_uv": (C.c_int, common[:5] + [C.c_double, C.c_double,
                                                    P(abi.gg_ray_out_t)]),
            "ggo_metric_tensor": (C.c_int, [P(abi.gg_metric_t), C.c_void_p, C.c_void_p]),
            "ggo_christoffel": (C.c_int, [P(abi.gg_metric_t), C.c_void_p, C.c_void_p]),
            "ggo_numerical_christoffel": (C.c_int, [P(abi.gg_metric_t), C.c_void_p,
                                                    C.c_double, C.c_void_p]),
            "ggo_geodesic_acceleration": (C.c_int, [P(abi.gg_metric_t), C.c_void_p,
                                                    C.c_void_p, C.c_void_p]),
            "ggo_event_horizon": (C.c_int, [P(abi.gg_metric_t), P(C.c_double)]),
            "ggo_orbital_four_velocity": (C.c_int, [P(abi.gg_metric_t), C.c_void_p,
                                                    C.c_void_p]),
            "ggo_rk4_run": (C.c_int, [P(abi.gg_metric_t), C.c_void_p, C.c_double,
                                      C.c_uint64]),
            "ggo_rk45_step": (C.c_int, [P(abi.gg_metric_t), P(abi.gg_integrator_t),
                                        C.c_void_p, P(C.c_double), P(C.c_int)]),
            "ggo_count_attempt_ops": (C.c_int, [P(abi.gg_metric_t), P(abi.gg_integrator_t),
                                                C.c_void_p, C.c_double, C.c_void_p]),
            "ggo_pixel_direction": (None, [P(abi.gg_camera_t), C.c_double, C.c_double,
                                           C.c_void_p]),
            "ggo_from_camera": (C.c_int, [P(abi.gg_metric_t), P(abi.gg_camera_t), C.c_uint32,
                                          C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p]),
            "ggo_redshift_factor": (C.c_double, [P(abi.gg_metric_t), C.c_void_p, C.c_void_p,
                                                 C.c_double]),
            "ggo_procedural_sky": (None, [C.c_void_p, C.c_void_p]),
            "ggo_spatial_dir": (None, [C.c_void_p, C.c_void_p]),
            "ggo_procedural_sky_n": (None, [C.c_void_p, C.c_void_p, C.c_uint64]),
            "ggo_from_camera_n": (C.c_int, [P(abi.gg_metric_t), P(abi.gg_camera_t), C.c_uint32,
                                            C.c_uint32, C.c_void_p, C.c_uint64, C.c_void_p]),
            "ggo_spatial_dir_n": (None, [C.c_void_p, C.c_void_p, C.c_uint64]),
            "ggo_checker_sky": (None, [C.c_double, C.c_double, C.c_uint32, C.c_uint32,
                                       C.c_uint64, C.c_void_p]),
            "ggo_disk_color": (None, [C.c_double, C.c_void_p]),
            "ggo_set_hdri": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_float]),
            "ggo_hdri_sky": (None, [C.c_void_p, C.c_void_p]),
            "ggo_set_scene": (C.c_int, [P(abi.gg_prim_t), C.c_uint32]),
            "ggo_scene_hit": (C.c_int, [C.c_void_p, C.c_void_p, P(C.c_double), C.c_void_p]),
            "ggo_encode_srgb": (None, [C.c_void_p, C.c_void_p]),
            "ggo_splitmix64": (C.c_uint64, [C.c_uint64]),
            "ggo_sample_uv": (None, [P(abi.gg_render_opts_t), C.c_uint32, C.c_uint32,
                                     C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p]),
            "ggo_kerr_isco": (C.c_double, [C.c_double, C.c_double]),
            "ggo_kerr_photon_orbit": (C.c_double, [C.c_double, C.c_double]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _LIBS[path] = L
    return _LIBS[path]


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


from gargantua_b200.curved import RayOutputs as RayArrays  # noqa: E402


def set_hdri(sky, variant: str = "plain") -> None:
    """Makes `sky` (a gargantua_b200.curved.HdriSky) the map of GG_SKY_HDRI renders."""
    px = np.ascontiguousarray(sky.pixels, np.float32)
    if lib(variant).ggo_set_hdri(_ptr(px), px.shape[1], px.shape[0], C.c_float(sky.intensity)):
        raise ValueError("empty sky map")


def hdri_sample(sky, direction) -> np.ndarray:
    """HdriSky::sample (sky.rs:108-122) of `sky` at a direction (3 floats)."""
    set_hdri(sky)
    d = np.ascontiguousarray(direction, np.float64)
    out = np.zeros(3)
    lib().ggo_hdri_sky(_ptr(d), _ptr(out))
    return out


def set_objects(objects, variant: str = "plain") -> None:
    """Makes `objects` (gargantua_b200.curved.SceneObjects) the scene of opts.scene renders."""
    arr = objects.to_c()
    if lib(variant).ggo_set_scene(arr, len(arr)):
        raise ValueError("unknown primitive kind or material")


def scene_hit(objects, origin, direction):
    """(index or -1, t, shaded colour) of the chord origin + t direction, t in (0, 1)."""
    set_objects(objects)
    o = np.ascontiguousarray(origin, np.float64)
    d = np.ascontiguousarray(direction, np.float64)
    t = C.c_double(0.0)
    rgb = np.zeros(3)
    k = lib().ggo_scene_hit(_ptr(o), _ptr(d), C.byref(t), _ptr(rgb))
    return k, t.value, rgb


def _sky_map(scene, variant: str) -> None:
    from gargantua_b200.curved import HdriSky
    if isinstance(scene.options.sky, HdriSky):
        set_hdri(scene.options.sky, variant)
    if scene.objects is not None:
        set_objects(scene.objects, variant)


def render(scene, threads: int = 0, rays: bool = True, variant: str = "plain"):
    """Render ``scene`` (a ``gargantua_b200.curved.Scene``) on the CPU oracle.

    Returns (rgb uint8 [H, W, 3], RayArrays or None)."""
    w, h = scene.width, scene.height
    n = w * h * scene.spp
    img = np.zeros((h, w, 3), np.uint8)
    ra = RayArrays(n) if rays else None
    _sky_map(scene, variant)
    st = lib(variant).ggo_render(*scene.c_args(), _ptr(img), C.byref(ra.struct()) if ra else None,
                          threads)
    abi.check(st, "ggo_render")
    return img, ra


def trace_samples(scene, index: np.ndarray, threads: int = 0,
                  variant: str = "plain") -> RayArrays:
    index = np.ascontiguousarray(index, np.uint64)
    ra = RayArrays(len(index))
    _sky_map(scene, variant)
    st = lib(variant).ggo_trace_samples(*scene.c_args(), _ptr(index), len(index),
                                 C.byref(ra.struct()), threads)
    abi.check(st, "ggo_trace_samples")
    return ra


def trace_uv(scene, u: float, v: float) -> RayArrays:
    ra = RayArrays(1)
    _sky_map(scene, "plain")
    st = lib().ggo_trace_uv(*scene.c_args()[:5], u, v, C.byref(ra.struct()))
    abi.check(st, "ggo_trace_uv")
    return ra


def sample_uv(scene, index: int) -> tuple[float, float]:
    spp = scene.spp
    pix, s = divmod(int(index), spp)
    py, px = divmod(pix, scene.width)
    uv = np.zeros(2)
    o = scene.options.to_c()
    lib().ggo_sample_uv(C.byref(o), scene.width, scene.height, px, py, s, _ptr(uv))
    return float(uv[0]), float(uv[1])


def near_class_boundary(scene, index: int, margin_m: float = 1e-6) -> bool:
    """True when re-shooting sample `index` with its image-plane point moved by
    an impact-parameter offset of `margin_m` (in units of M) in +-u or +-v
    changes its termination class: the sample lies on a class boundary."""
    u, v = sample_uv(scene, index)
    cam = scene.camera
    half_h = np.tan(cam.fov_y_radians / 2.0)
    half_w = half_h * cam.aspect
    r_cam = cam.position[1]
    du = margin_m / (r_cam * half_w)
    dv = margin_m / (r_cam * half_h)
    base = trace_uv(scene, u, v).cls[0]
    for uu, vv in ((u + du, v), (u - du, v), (u, v + dv), (u, v - dv)):
        if trace_uv(scene, uu, vv).cls[0] != base:
            return True
    return False


def trace_cross(scene, index: np.ndarray, threads: int = 0) -> np.ndarray:
    index = np.ascontiguousarray(index, np.uint64)
    out = np.zeros((8, len(index)), np.float64)
    st = lib().ggo_trace_cross(*scene.c_args(), _ptr(index), len(index), _ptr(out), threads)
    abi.check(st, "ggo_trace_cross")
    return out


def kerr_thin_1080p():
    """The Kerr a = 0.9 1920x1080 thin-disk frame (camera r = 50 M at 75 deg,
    60 deg FOV, disk r_ISCO-30 M with q = 3, 18x36 checkerboard sky seed 0,
    the reference's RK45 step with rtol 1e-8 / atol 1e-10, 10,000 step()
    calls, escape at 200 M), built from the oracle alone: the ISCO from
    ``ggo_kerr_isco`` and the camera frame written out here, so that timing
    the oracle on it maps none of the product's native code.  Field for field
    the scene ``gargantua_b200.workloads.kerr_thin_1080p()`` builds (a test
    checks that)."""
    import math

    from gargantua_b200.curved import Camera, CheckerSky, RenderOptions, Scene, ThinDisk
    from gargantua_b200.gr_core import Kerr, RK45Integrator

    k = Kerr(1.0, 0.9)
    incl = math.radians(75.0)
    cam = Camera((0.0, 50.0, incl, 0.0), (-math.sin(incl), 0.0, -math.cos(incl)),
                 (0.0, 0.0, 1.0), math.radians(60.0), 1920 / 1080)
    integ = RK45Integrator(max_radius=200.0, rtol=1e-8, atol=1e-10)
    return Scene(k, cam, 1920, 1080, ThinDisk(lib().ggo_kerr_isco(k.mass, k.spin), 30.0, 3.0),
                 RenderOptions(sky=CheckerSky(18, 36, 0), max_steps=10000, integrator=integ))


def procedural_sky_n(dirs: np.ndarray) -> np.ndarray:
    """ProceduralSky::sample (sky.rs:26-40) of n directions (n x 3) -> n x 3."""
    d = np.ascontiguousarray(dirs, np.float64)
    out = np.zeros_like(d)
    lib().ggo_procedural_sky_n(_ptr(d), _ptr(out), len(d))
    return out


def spatial_dir_n(vel: np.ndarray) -> np.ndarray:
    """spatial_dir (tracer.rs:185-189) of n velocities (n x 4) -> n x 3."""
    v = np.ascontiguousarray(vel, np.float64)
    out = np.zeros((len(v), 3))
    lib().ggo_spatial_dir_n(_ptr(v), _ptr(out), len(v))
    return out


def initial_states(scene, index: np.ndarray | None = None) -> tuple[np.ndarray, np.ndarray]:
    """GeodesicRay::from_camera (ray.rs:14-61) at the centres of pixels
    `index` (py * width + px; default all): positions and velocities, 4 x n
    each."""
    idx = np.arange(scene.width * scene.height, dtype=np.uint64) if index is None else \
        np.ascontiguousarray(index, np.uint64)
    st = np.zeros((len(idx), 9))
    m, c = scene.metric.to_c(), scene.camera.to_c()
    r = lib().ggo_from_camera_n(C.byref(m), C.byref(c), scene.width, scene.height, _ptr(idx),
                                len(idx), _ptr(st))
    abi.check(r, "ggo_from_camera_n")
    return st[:, :4].T.copy(), st[:, 4:8].T.copy()
