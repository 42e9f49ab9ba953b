"""ctypes mirror of ``include/gargantua_gpu.h`` and the loader of the CUDA library.

The structs below are field-for-field copies of the C header's POD structs;
``gg_struct_size`` in the library is compared against ``ctypes.sizeof`` by the
tests, so a drift between the two fails loudly.

The library is ``gargantua_b200/libgargantua_gpu.so``, built in-tree by
``gargantua_b200/build.py``.  There is no fallback: if it is missing,
``load()`` raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "libgargantua_gpu.so"

GG_OK = 0
GG_ERR_INVALID_ARG = -1
GG_ERR_CUDA = -2
GG_ERR_OOM = -3
GG_ERR_BUDGET = -4
GG_ERR_UNSUPPORTED = -5
GG_ERR_NO_DEVICE = -6
GG_ERR_TOO_LARGE = -7

GG_METRIC_SCHWARZSCHILD = 0
GG_METRIC_KERR = 1
GG_DISK_NONE = 0
GG_DISK_VOLUMETRIC = 1
GG_DISK_THIN = 2
GG_PREC_FP64 = 0
GG_PREC_MIXED = 1
GG_STEPPER_REFERENCE = 0
GG_STEPPER_DP45 = 1
GG_BATCH_VARIANTS = 12


def batch_variant(v: int) -> tuple[int, int, int, int]:
    """(refill period, CTAs per SM, threads per CTA, samples per queue claim)
    of batch kernel variant v (gg_batch_variant_info)."""
    out = (C.c_int32 * 4)()
    check(load().gg_batch_variant_info(int(v), out), "gg_batch_variant_info")
    return tuple(out)


def batch_variant_names() -> list[str]:
    """The batch kernel variants gg_batch_autotune chooses from, by index."""
    return ["period {}, {} CTAs/SM, {} threads, chunk {}".format(*batch_variant(v))
            for v in range(GG_BATCH_VARIANTS)]
GG_SKY_PROCEDURAL = 0
GG_SKY_CHECKER = 1
GG_SKY_HDRI = 2

GG_CLASS_HORIZON = 0
GG_CLASS_ESCAPED = 1
GG_CLASS_DISK = 2
GG_CLASS_MAXSTEPS = 3
GG_CLASS_BUDGET = 4
GG_CLASS_SCENE = 5
GG_N_CLASSES = 6

GG_PRIM_SPHERE = 0
GG_PRIM_QUAD = 1
GG_MAT_LAMBERTIAN = 0
GG_MAT_DIFFUSE_LIGHT = 1
GG_MAT_METAL = 2
GG_MAT_DIELECTRIC = 3


class gg_metric_t(C.Structure):
    _fields_ = [("kind", C.c_int32), ("reserved", C.c_int32), ("mass", C.c_double),
                ("spin", C.c_double)]


class gg_camera_t(C.Structure):
    _fields_ = [("position", C.c_double * 4), ("look_at", C.c_double * 3),
                ("up", C.c_double * 3), ("fov_y_radians", C.c_double), ("aspect", C.c_double)]


class gg_disk_t(C.Structure):
    _fields_ = [("kind", C.c_int32), ("reserved", C.c_int32), ("r_inner", C.c_double),
                ("r_outer", C.c_double), ("scale_height", C.c_double),
                ("density_0", C.c_double), ("temperature_0", C.c_double),
                ("emissivity_index", C.c_double)]


class gg_integrator_t(C.Structure):
    _fields_ = [("initial_step", C.c_double), ("min_step", C.c_double),
                ("max_step", C.c_double), ("tolerance", C.c_double),
                ("max_radius", C.c_double), ("horizon_buffer", C.c_double),
                ("rtol", C.c_double), ("atol", C.c_double), ("max_steps", C.c_uint32),
                ("precision", C.c_int32), ("stepper", C.c_int32), ("reserved", C.c_int32)]


class gg_render_opts_t(C.Structure):
    _fields_ = [("samples_per_axis", C.c_uint32), ("jitter_spp", C.c_uint32),
                ("seed", C.c_uint64), ("sky", C.c_int32), ("sky_rows", C.c_uint32),
                ("sky_cols", C.c_uint32), ("row_offset", C.c_uint32), ("sky_seed", C.c_uint64),
                ("attempt_budget", C.c_uint64), ("row_step", C.c_uint32), ("scene", C.c_uint32)]


class gg_ray_out_t(C.Structure):
    _fields_ = [("cls", C.POINTER(C.c_int32)), ("x", C.POINTER(C.c_double)),
                ("v", C.POINTER(C.c_double)), ("lambda_", C.POINTER(C.c_double)),
                ("attempts", C.POINTER(C.c_uint32)), ("accepted", C.POINTER(C.c_uint32)),
                ("intensity", C.POINTER(C.c_double)), ("color_temp", C.POINTER(C.c_double)),
                ("rgb", C.POINTER(C.c_double)), ("cross", C.POINTER(C.c_double))]


class gg_scene_t(C.Structure):
    _fields_ = [("metric", gg_metric_t), ("camera", gg_camera_t), ("disk", gg_disk_t),
                ("width", C.c_uint32), ("height", C.c_uint32), ("sky_seed", C.c_uint64)]


class gg_stats_t(C.Structure):
    _fields_ = [("rays", C.c_uint64), ("attempts", C.c_uint64), ("accepted", C.c_uint64),
                ("class_count", C.c_uint64 * GG_N_CLASSES), ("kernel_ms", C.c_double),
                ("fp64_rays", C.c_uint64), ("fp64_attempts", C.c_uint64)]


class gg_prim_t(C.Structure):
    _fields_ = [("kind", C.c_int32), ("material", C.c_int32), ("p", C.c_double * 3),
                ("u", C.c_double * 3), ("v", C.c_double * 3), ("radius", C.c_double),
                ("color", C.c_double * 3), ("fuzz", C.c_double), ("ior", C.c_double)]


STRUCTS = {
    "gg_metric_t": gg_metric_t,
    "gg_camera_t": gg_camera_t,
    "gg_disk_t": gg_disk_t,
    "gg_integrator_t": gg_integrator_t,
    "gg_render_opts_t": gg_render_opts_t,
    "gg_ray_out_t": gg_ray_out_t,
    "gg_scene_t": gg_scene_t,
    "gg_stats_t": gg_stats_t,
    "gg_prim_t": gg_prim_t,
}

P = C.POINTER
_SIGNATURES = {
    "gg_version": (C.c_char_p, []),
    "gg_strerror": (C.c_char_p, [C.c_int]),
    "gg_struct_size": (C.c_int, [C.c_char_p]),
    "gg_metric_schwarzschild": (C.c_int, [P(gg_metric_t), C.c_double]),
    "gg_metric_kerr": (C.c_int, [P(gg_metric_t), C.c_double, C.c_double]),
    "gg_integrator_default": (None, [P(gg_integrator_t)]),
    "gg_disk_default": (None, [P(gg_disk_t)]),
    "gg_render_opts_default": (None, [P(gg_render_opts_t)]),
    "gg_camera_inclined": (C.c_int, [P(gg_camera_t), C.c_double, C.c_double, C.c_double,
                                     C.c_double]),
    "gg_kerr_isco": (C.c_double, [C.c_double, C.c_double]),
    "gg_kerr_photon_orbit": (C.c_double, [C.c_double, C.c_double]),
    "gg_validate": (C.c_int, [P(gg_metric_t), P(gg_camera_t), P(gg_disk_t),
                              P(gg_integrator_t), P(gg_render_opts_t), C.c_uint32,
                              C.c_uint32]),
    "gg_create": (C.c_int, [P(C.c_void_p), C.c_int]),
    "gg_destroy": (C.c_int, [C.c_void_p]),
    "gg_stream": (C.c_void_p, [C.c_void_p]),
    "gg_last_stats": (C.c_int, [C.c_void_p, P(gg_stats_t)]),
    "gg_render": (C.c_int, [C.c_void_p, P(gg_metric_t), P(gg_camera_t), P(gg_disk_t),
                            P(gg_integrator_t), P(gg_render_opts_t), C.c_uint32, C.c_uint32,
                            C.c_void_p, P(gg_ray_out_t)]),
    "gg_render_device": (C.c_int, [C.c_void_p, P(gg_metric_t), P(gg_camera_t), P(gg_disk_t),
                                   P(gg_integrator_t), P(gg_render_opts_t), C.c_uint32,
                                   C.c_uint32, C.c_void_p, P(gg_ray_out_t), C.c_void_p]),
    "gg_measure_fma_peak": (C.c_int, [C.c_void_p, C.c_int, P(C.c_double)]),
    "gg_polar_sincos": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32]),
    "gg_check_procedural_sky": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p]),
    "gg_check_spatial_dir": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p]),
    "gg_check_kerr_vjp": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_int, C.c_void_p]),
    "gg_check_step_factor": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p]),
    "gg_render_batch": (C.c_int, [C.c_void_p, P(gg_scene_t), C.c_uint32, P(gg_integrator_t),
                                  P(gg_render_opts_t), C.c_void_p]),
    "gg_render_batch_device": (C.c_int, [C.c_void_p, P(gg_scene_t), C.c_uint32,
                                         P(gg_integrator_t), P(gg_render_opts_t), C.c_void_p,
                                         C.c_void_p]),
    "gg_batch_autotune": (C.c_int, [C.c_void_p, P(gg_scene_t), C.c_uint32, P(gg_integrator_t),
                                    P(gg_render_opts_t), P(C.c_int), P(C.c_double)]),
    "gg_batch_set_variant": (C.c_int, [C.c_void_p, C.c_int]),
    "gg_batch_variant_info": (C.c_int, [C.c_int, C.c_void_p]),
    "gg_set_hdri": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_float]),
    "gg_set_scene": (C.c_int, [C.c_void_p, P(gg_prim_t), C.c_uint32]),
    "gg_scene_validate": (C.c_int, [P(gg_prim_t), C.c_uint32, P(C.c_uint32), P(C.c_uint32)]),
    "gg_forward_ckpt": (C.c_int, [C.c_void_p, P(gg_metric_t), C.c_double, C.c_double, C.c_double,
                                  C.c_double, P(gg_disk_t), P(gg_integrator_t),
                                  P(gg_render_opts_t), C.c_uint32, C.c_uint32, C.c_void_p,
                                  C.c_void_p]),
    "gg_backward": (C.c_int, [C.c_void_p, C.c_void_p, P(C.c_double), C.c_void_p]),
    "gg_render_device_noalloc": (C.c_int, [P(gg_metric_t), P(gg_camera_t), P(gg_disk_t),
                                           P(gg_integrator_t), P(gg_render_opts_t), C.c_uint32,
                                           C.c_uint32, C.c_void_p, P(gg_ray_out_t),
                                           C.c_void_p]),
}


class GargantuaError(RuntimeError):
    """A non-zero status from the C ABI."""

    def __init__(self, status: int, where: str, message: str):
        super().__init__(f"{where}: {message} (status {status})")
        self.status = status


_LIB = None


def load(path: os.PathLike | str | None = None) -> C.CDLL:
    """Load ``libgargantua_gpu.so`` and attach the C signatures.  Raises if absent."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = Path(path) if path is not None else LIB_PATH
    if not p.exists():
        raise FileNotFoundError(
            f"{p} is missing: build it with `python -m gargantua_b200.build` "
            "(there is no CPU fallback)")
    lib = C.CDLL(str(p))
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _LIB = lib
    return lib


def check(status: int, where: str) -> None:
    if status != GG_OK:
        msg = load().gg_strerror(status).decode()
        raise GargantuaError(status, where, msg)


def header_functions(header: os.PathLike | str | None = None) -> list[str]:
    """Names of every GG_API function the C header declares."""
    import re
    h = Path(header) if header else PKG_DIR.parent / "include" / "gargantua_gpu.h"
    text = h.read_text()
    return re.findall(r"GG_API\s+[\w\s\*]+?\b(gg_\w+)\s*\(", text)
