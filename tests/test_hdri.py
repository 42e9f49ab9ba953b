"""The equirectangular sky map (HdriSky, crates/raytracer/src/curved/sky.rs:43-123)
and the Radiance .hdr files it is read from.

CPU: the oracle's restatement against the reference's three sky tests
(sky.rs:133-163) and hand-worked texel lookups; the .hdr reader against the
writer (flat, adaptive and old run-length scanlines) and the RGBE decoding
rule; argument checks.  GPU: the map sampled by the kernels equals the
oracle's sample at each escaped ray's own final direction (the device and
host acos / atan2 may differ in the last bit, so the bar is 1e-6 absolute,
bit-equal on 99.9 % of rays), and whole images match the oracle's.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from gargantua_b200 import abi, hdr, workloads
from gargantua_b200.curved import HdriSky, RenderOptions
from gargantua_b200.gr_core import Kerr


# ---- reference tests, restated on the oracle ----------------------------
def test_constant_color(oracle_mod):  # sky.rs:133-141
    sky = HdriSky.from_pixels(4, 2, [[0.4, 0.6, 0.8]] * 8)
    c = oracle_mod.hdri_sample(sky, (1.0, 0.0, 0.0))
    assert np.all(np.abs(c - [0.4, 0.6, 0.8]) < 1e-4)


def test_pole_is_top_row(oracle_mod):  # sky.rs:143-153
    px = np.zeros((2, 4, 3), np.float32)
    px[0] = [1.0, 0.0, 0.0]
    px[1] = [0.0, 0.0, 1.0]
    sky = HdriSky(px)
    top = oracle_mod.hdri_sample(sky, (0.0, 0.0, 1.0))
    assert top[0] > 0.9 and top[2] < 0.1
    bot = oracle_mod.hdri_sample(sky, (0.0, 0.0, -1.0))
    assert bot[2] > 0.9 and bot[0] < 0.1


def test_intensity_scales(oracle_mod):  # sky.rs:155-162
    sky = HdriSky.from_pixels(2, 2, [[0.5, 0.25, 0.1]] * 4).with_intensity(2.0)
    c = oracle_mod.hdri_sample(sky, (1.0, 0.0, 0.0))
    assert abs(c[0] - 1.0) < 1e-4 and abs(c[1] - 0.5) < 1e-4


def _numbered(w, h):
    """Texel (y, x) holds (y, x, 10 y + x)."""
    px = np.zeros((h, w, 3), np.float32)
    for y in range(h):
        for x in range(w):
            px[y, x] = (y, x, 10 * y + x)
    return px


@pytest.mark.parametrize("direction,want", [
    # +y: phi = pi/2 -> u = 3/4, fx = 3; theta = pi/2 -> v = 1/2, fy = 1:
    # texel (1, 3) exactly
    ((0.0, 1.0, 0.0), (1.0, 3.0, 13.0)),
    # -x: phi = pi -> u = 1, fx = 4 rem 4 = 0; texel (1, 0)
    ((-1.0, 0.0, 0.0), (1.0, 0.0, 10.0)),
    # +x: u = 1/2, fx = 2; texel (1, 2)
    ((1.0, 0.0, 0.0), (1.0, 2.0, 12.0)),
    # -z: fy = 2 clamped to h - 1 = 1, x = 2: texel (1, 2), y1 clamped
    ((0.0, 0.0, -1.0), (1.0, 2.0, 12.0)),
    # +z: fy = 0, row 0, x = 2 (phi = atan2(0, 0) = 0)
    ((0.0, 0.0, 1.0), (0.0, 2.0, 2.0)),
])
def test_texel_centres(oracle_mod, direction, want):
    sky = HdriSky(_numbered(4, 2))
    got = oracle_mod.hdri_sample(sky, direction)
    assert np.array_equal(got, np.array(want)), got


def test_bilinear_and_wrap(oracle_mod):
    sky = HdriSky(_numbered(4, 3))
    # x0 = 3 and x1 wraps to 0
    phi = np.pi - 0.5 * (2 * np.pi / 4)  # u = 7/8, fx = 3.5
    theta = np.pi * (1.25 / 3)            # fy = 1.25
    d = (np.sin(theta) * np.cos(phi), np.sin(theta) * np.sin(phi), np.cos(theta))
    got = oracle_mod.hdri_sample(sky, d)
    # y: 1 + 0.25; x: lerp(3, 0, 0.5) = 1.5; third: lerp rows of lerp(10y+3, 10y, 0.5)
    assert np.allclose(got, [1.25, 1.5, 10 * 1.25 + 1.5], atol=2e-5), got


# ---- .hdr files ---------------------------------------------------------
def test_rgbe_decoding_rule():
    rgbe = np.array([[128, 64, 0, 129], [255, 1, 2, 0], [1, 2, 3, 136]], np.uint8)
    got = hdr.rgbe_to_float(rgbe)
    assert np.array_equal(got[0], np.float32([128 / 128, 64 / 128, 0.0]))
    assert np.array_equal(got[1], np.zeros(3, np.float32))
    assert np.array_equal(got[2], np.float32([1, 2, 3]))


@pytest.mark.parametrize("w,h,rle", [(37, 5, True), (37, 5, False), (5, 3, True), (300, 2, True)])
def test_hdr_round_trip(tmp_path, w, h, rle):
    rng = np.random.default_rng(w * 100 + h)
    rgb = (rng.random((h, w, 3)) * 10.0 ** rng.integers(-3, 3, (h, w, 1))).astype(np.float32)
    rgb[0, : w // 2] = rgb[0, 0]  # runs for the run-length coder
    rgb[h - 1, 1] = 0.0
    path = tmp_path / "m.hdr"
    hdr.write_hdr(path, rgb, rle=rle)
    got = hdr.read_hdr(path)
    assert got.shape == (h, w, 3) and got.dtype == np.float32
    assert np.array_equal(got, hdr.rgbe_to_float(hdr.float_to_rgbe(rgb)))
    # RGBE keeps 8 mantissa bits of the largest channel
    m = rgb.max(axis=2, keepdims=True)
    assert np.all(np.abs(got - rgb) <= m * 2.0 ** -7 + 1e-30)
    sky = HdriSky.from_file(path)
    assert (sky.width, sky.height) == (w, h)


def test_hdr_old_run_length():
    head = b"#?RGBE\n\n-Y 1 +X 6\n"
    body = bytes((10, 20, 30, 130)) + bytes((1, 1, 1, 3)) + bytes((5, 6, 7, 128)) + \
        bytes((1, 1, 1, 1))
    got = hdr.decode_hdr(head + body)
    want = hdr.rgbe_to_float(np.array([[10, 20, 30, 130]] * 4 + [[5, 6, 7, 128]] * 2, np.uint8))
    assert np.array_equal(got[0], want)


@pytest.mark.parametrize("data", [
    b"P6\n",
    b"#?RADIANCE\nFORMAT=32-bit_rle_xyze\n\n-Y 1 +X 1\n\x00\x00\x00\x00",
    b"#?RADIANCE\n\n+Y 1 +X 1\n\x00\x00\x00\x00",
    b"#?RADIANCE\n\n-Y 1 +X 2\n\x00\x00\x00\x00",
    b"#?RADIANCE\n\n-Y 1 +X 8\n\x02\x02\x00\x08\x88",
])
def test_hdr_rejects_malformed(data):
    with pytest.raises(ValueError):
        hdr.decode_hdr(data)


# ---- interface ------------------------------------------------------------
def test_python_sky_and_options():
    with pytest.raises(ValueError):
        HdriSky.from_pixels(3, 2, [[0.0, 0.0, 0.0]] * 5)
    with pytest.raises(ValueError):
        HdriSky(np.zeros((2, 3), np.float32))
    sky = HdriSky(np.ones((2, 4, 3)), 1.5)
    o = RenderOptions(sky=sky).to_c()
    assert o.sky == abi.GG_SKY_HDRI
    k = sky.key()
    sky.with_intensity(2.0)
    assert sky.key() != k


def test_validate_accepts_the_map_kind(gglib):
    scene = workloads.schwarzschild_thin_256()
    scene.options = RenderOptions(sky=HdriSky(np.ones((2, 4, 3))), max_steps=5000,
                                  integrator=scene.options.integrator)
    assert gglib.gg_validate(*scene.c_args()) == abi.GG_OK
    o = scene.options.to_c()
    o.sky = 3
    m, c, d, i, _ = scene.c_structs()
    assert gglib.gg_validate(C.byref(m), C.byref(c), C.byref(d), C.byref(i), C.byref(o),
                             scene.width, scene.height) == abi.GG_ERR_INVALID_ARG


# ---- GPU ------------------------------------------------------------------
def _map(seed=3, w=37, h=19):
    rng = np.random.default_rng(seed)
    return HdriSky((rng.random((h, w, 3)) * 2.0).astype(np.float32), 1.7)


def _with_sky(scene, sky):
    scene.options.sky = sky
    return scene


def _sky_of_final_velocity(oracle_mod, sky, v):
    """The oracle's map sample at spatial_dir of each final velocity (tracer.rs:185-189)."""
    s = v[1:4].T
    n = np.sqrt(s[:, 0] * s[:, 0] + s[:, 1] * s[:, 1] + s[:, 2] * s[:, 2])
    d = s / n[:, None]
    oracle_mod.set_hdri(sky)
    out = np.zeros((len(d), 3))
    L = oracle_mod.lib()
    for k in range(len(d)):
        dk = np.ascontiguousarray(d[k])
        L.ggo_hdri_sky(dk.ctypes.data_as(C.c_void_p), out[k].ctypes.data_as(C.c_void_p))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["fp64", "mixed"])
def test_map_sample_equals_oracle(renderer, oracle_mod, form):
    sky = _map()
    if form == "mixed":
        scene = workloads.kerr_thin_1080p(precision=abi.GG_PREC_MIXED,
                                          stepper=abi.GG_STEPPER_DP45)
        scene.width, scene.height = 320, 180
    else:
        scene = workloads.schwarzschild_thin_256()
    _with_sky(scene, sky)
    _, g = renderer.render(scene, rays=True)
    esc = np.flatnonzero(g.cls == 1)
    assert len(esc) > 5000
    want = _sky_of_final_velocity(oracle_mod, sky, g.v[:, esc])
    got = g.rgb[esc]
    assert np.abs(got - want).max() <= 1e-6
    assert (got == want).all(axis=1).mean() >= 0.999


@pytest.mark.gpu
def test_map_render_matches_oracle_image(renderer, oracle_mod):
    scene = _with_sky(workloads.schwarzschild_thin_256(), _map(5, 64, 32))
    img, _ = renderer.render(scene)
    oimg, _ = oracle_mod.render(scene, rays=False)
    assert (img == oimg).all(axis=2).mean() > 0.9999
    # a new map object re-uploads; the same object with a new intensity too
    dim = HdriSky(scene.options.sky.pixels, 0.25)
    img2, _ = renderer.render(_with_sky(scene, dim))
    assert img2.astype(int).sum() < img.astype(int).sum()
    dim.with_intensity(1.7)
    img3, _ = renderer.render(scene)
    assert np.array_equal(img3, img)


@pytest.mark.gpu
def test_map_kind_without_a_map_and_unsupported_paths(gglib):
    from gargantua_b200.curved import Renderer
    r = Renderer(0)
    try:
        scene = _with_sky(workloads.schwarzschild_thin_256(), _map())
        img = np.zeros((scene.height, scene.width, 3), np.uint8)
        st = gglib.gg_render(r.handle, *scene.c_args(), img.ctypes.data_as(C.c_void_p), None)
        assert st == abi.GG_ERR_INVALID_ARG
        assert gglib.gg_set_hdri(r.handle, None, 4, 2, C.c_float(1.0)) == abi.GG_ERR_INVALID_ARG
        px = np.ones((2, 4, 3), np.float32)
        assert gglib.gg_set_hdri(r.handle, px.ctypes.data_as(C.c_void_p), 0, 2,
                                 C.c_float(1.0)) == abi.GG_ERR_INVALID_ARG
        st = gglib.gg_render_device_noalloc(*scene.c_args(), None, None, None)
        assert st == abi.GG_ERR_UNSUPPORTED
        b = workloads.batch_scenes(2, max_side=64)
        for s in b:
            s.options.sky = scene.options.sky
        with pytest.raises(Exception):
            r.render_batch(b)
    finally:
        r.close()


@pytest.mark.gpu
def test_map_kerr_volumetric(renderer, oracle_mod):
    """The map behind the volumetric disk (render_with_disk)."""
    sky = _map(7, 48, 24)
    scene = workloads.schwarzschild_thin_256()
    scene.metric = Kerr(1.0, 0.6)
    from gargantua_b200.curved import AccretionDisk
    # the density is nonzero on the whole cylindrical shell r_in <= R <= r_out
    # at any height, so only rays passing outside R = 8 M escape
    scene.disk = AccretionDisk(r_inner=6.0, r_outer=8.0)
    scene.width = scene.height = 96
    _with_sky(scene, sky)
    _, g = renderer.render(scene, rays=True)
    esc = np.flatnonzero(g.cls == 1)
    assert len(esc) > 1000
    want = _sky_of_final_velocity(oracle_mod, sky, g.v[:, esc])
    assert np.abs(g.rgb[esc] - want).max() <= 1e-6
