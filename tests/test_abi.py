"""The C ABI on the CPU: the library loads, exports every declared symbol, its
struct layouts match the ctypes mirror, and the host-only entry points
(constructors, defaults, validation) behave as documented.  No compute call
runs here; that needs an sm_100 device (tests marked gpu)."""
from __future__ import annotations

import ctypes as C
import math

import pytest

from gargantua_b200 import abi
from gargantua_b200.curved import Camera, RenderOptions, Scene, ThinDisk
from gargantua_b200.gr_core import Kerr, Schwarzschild


def test_every_declared_function_is_exported(gglib):
    names = abi.header_functions()
    assert len(names) >= 18
    for n in names:
        assert hasattr(gglib, n), n
        assert n in abi._SIGNATURES, f"{n} missing from the ctypes mirror"


def test_struct_layouts_match(gglib):
    for name, cls in abi.STRUCTS.items():
        assert gglib.gg_struct_size(name.encode()) == C.sizeof(cls), name
    assert gglib.gg_struct_size(b"nope") == -1


def test_strerror_covers_codes(gglib):
    for code in (0, -1, -2, -3, -4, -5, -6):
        assert gglib.gg_strerror(code).decode() not in ("", "unknown status")
    assert gglib.gg_strerror(-99).decode() == "unknown status"
    assert b"sm_100a" in gglib.gg_version()


def test_metric_constructors(gglib):
    m = abi.gg_metric_t()
    assert gglib.gg_metric_kerr(C.byref(m), 1.0, 1.2) == abi.GG_OK
    assert m.spin == pytest.approx(0.9999)
    assert gglib.gg_metric_kerr(C.byref(m), 0.0, 0.5) == abi.GG_ERR_INVALID_ARG
    assert gglib.gg_metric_kerr(C.byref(m), 1.0, float("nan")) == abi.GG_ERR_INVALID_ARG
    assert gglib.gg_metric_schwarzschild(C.byref(m), 2.0) == abi.GG_OK
    assert m.kind == abi.GG_METRIC_SCHWARZSCHILD and m.mass == 2.0
    assert gglib.gg_metric_schwarzschild(C.byref(m), -1.0) == abi.GG_ERR_INVALID_ARG


def test_defaults_match_reference(gglib):
    i = abi.gg_integrator_t()
    gglib.gg_integrator_default(C.byref(i))
    assert (i.initial_step, i.min_step, i.max_step, i.tolerance, i.max_radius,
            i.horizon_buffer, i.max_steps) == (0.1, 1e-8, 1.0, 1e-6, 200.0, 0.01, 5000)
    d = abi.gg_disk_t()
    gglib.gg_disk_default(C.byref(d))
    assert (d.r_inner, d.r_outer, d.scale_height, d.density_0, d.temperature_0) == \
        (6.0, 20.0, 1.0, 1.0, 1.0)
    o = abi.gg_render_opts_t()
    gglib.gg_render_opts_default(C.byref(o))
    assert o.samples_per_axis == 1 and o.sky == abi.GG_SKY_PROCEDURAL


def test_special_radii(gglib):
    assert gglib.gg_kerr_isco(1.0, 0.0) == pytest.approx(6.0, abs=1e-12)
    assert gglib.gg_kerr_isco(1.0, 0.9) == pytest.approx(2.320883041761887, abs=1e-12)
    assert gglib.gg_kerr_photon_orbit(1.0, 0.0) == pytest.approx(3.0, abs=1e-12)
    assert gglib.gg_kerr_photon_orbit(1.0, 0.9) == pytest.approx(1.5578546274233829, abs=1e-12)


def test_inclined_camera(gglib):
    c = Camera.inclined(30.0, math.radians(80.0), math.radians(60.0), 1.0)
    assert c.position[1] == 30.0 and c.position[2] == pytest.approx(math.radians(80.0))
    assert c.look_at[0] == pytest.approx(-math.sin(math.radians(80.0)))
    assert c.up == (0.0, 0.0, 1.0)


def _valid(scene):
    return abi.load().gg_validate(*scene.c_args())


def test_validation(gglib):
    ok = Scene(Kerr(1.0, 0.9), Camera.inclined(50.0, 1.3, 1.0, 16 / 9), 64, 36,
               ThinDisk(2.32, 30.0, 3.0), RenderOptions())
    assert _valid(ok) == abi.GG_OK
    bad = []
    s = Scene(Schwarzschild(1.0), Camera(), 0, 10)
    bad.append(s)
    s = Scene(Schwarzschild(1.0), Camera(position=(0.0, float("nan"), 1.0, 0.0)), 8, 8)
    bad.append(s)
    s = Scene(Schwarzschild(1.0), Camera(look_at=(0.0, 0.0, 1.0), up=(0.0, 0.0, 2.0)), 8, 8)
    bad.append(s)
    s = Scene(Schwarzschild(1.0), Camera(fov_y_radians=4.0), 8, 8)
    bad.append(s)
    s = Scene(Schwarzschild(1.0), Camera(), 8, 8, ThinDisk(10.0, 5.0, 3.0))
    bad.append(s)
    s = Scene(Schwarzschild(1.0), Camera(), 8, 8, None, RenderOptions(max_steps=0))
    bad.append(s)
    s = Scene(Schwarzschild(1.0), Camera(), 1 << 20, 1 << 20, None,
              RenderOptions(samples_per_axis=4))
    bad.append(s)
    for b in bad:
        assert _valid(b) == abi.GG_ERR_INVALID_ARG, b
    m = Schwarzschild(-1.0)
    assert _valid(Scene(m, Camera(), 8, 8)) == abi.GG_ERR_INVALID_ARG


def test_render_rejects_bad_args_before_touching_a_device(gglib):
    # a NULL context is refused without any CUDA call
    s = Scene(Schwarzschild(1.0), Camera(), 8, 8)
    assert gglib.gg_render(None, *s.c_args(), None, None) == abi.GG_ERR_INVALID_ARG


def test_no_device_is_reported():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    h = C.c_void_p()
    assert abi.load().gg_create(C.byref(h), 0) == abi.GG_ERR_NO_DEVICE
