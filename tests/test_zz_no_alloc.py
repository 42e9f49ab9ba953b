"""gg_render_device_noalloc: the render entry point for callers that cannot let
a library allocate device memory (an application-owned arena or pool, no
allocation after start-up, no cudaMalloc synchronisation).  Its scratch is a
fixed file-scope device array instead of context-owned buffers.

Checked through the C ABI against the context-based gg_render on the same
scenes, for two calls in a row (the shared scratch keeps the previous call's
contents, so the second call shows the counters are cleared), on a
supersampled scene that uses the array's colour buffer and on a single-sample
one.  Named so pytest collects it last; it also passes alone.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from gargantua_b200 import abi, workloads
from gargantua_b200.curved import RayOutputs, Renderer

pytestmark = pytest.mark.gpu

FIELDS = ("cls", "x", "v", "lam", "attempts", "accepted", "intensity", "color_temp", "rgb",
          "cross")


def device_rays(torch, n):
    t = {
        "cls": torch.zeros(n, dtype=torch.int32, device="cuda"),
        "x": torch.zeros(4 * n, dtype=torch.float64, device="cuda"),
        "v": torch.zeros(4 * n, dtype=torch.float64, device="cuda"),
        "lam": torch.zeros(n, dtype=torch.float64, device="cuda"),
        "attempts": torch.zeros(n, dtype=torch.int32, device="cuda"),
        "accepted": torch.zeros(n, dtype=torch.int32, device="cuda"),
        "intensity": torch.zeros(n, dtype=torch.float64, device="cuda"),
        "color_temp": torch.zeros(n, dtype=torch.float64, device="cuda"),
        "rgb": torch.zeros(3 * n, dtype=torch.float64, device="cuda"),
        "cross": torch.zeros(8 * n, dtype=torch.float64, device="cuda"),
    }

    def p(name, ct):
        return C.cast(C.c_void_p(t[name].data_ptr()), C.POINTER(ct))
    s = abi.gg_ray_out_t(p("cls", C.c_int32), p("x", C.c_double), p("v", C.c_double),
                         p("lam", C.c_double), p("attempts", C.c_uint32),
                         p("accepted", C.c_uint32), p("intensity", C.c_double),
                         p("color_temp", C.c_double), p("rgb", C.c_double),
                         p("cross", C.c_double))
    return t, s


def noalloc_render(torch, scene):
    lib = abi.load()
    n = scene.n_samples
    rgb = torch.zeros(scene.width * scene.height * 3, dtype=torch.uint8, device="cuda")
    rays, rs = device_rays(torch, n)
    stream = torch.cuda.current_stream()
    st = lib.gg_render_device_noalloc(*scene.c_args(), C.c_void_p(rgb.data_ptr()),
                                      C.byref(rs), C.c_void_p(stream.cuda_stream))
    assert st == abi.GG_OK, lib.gg_strerror(st)
    stream.synchronize()
    img = rgb.cpu().numpy().reshape(scene.height, scene.width, 3)
    out = RayOutputs(n)
    out.cls = rays["cls"].cpu().numpy()
    out.x = rays["x"].cpu().numpy().reshape(4, n)
    out.v = rays["v"].cpu().numpy().reshape(4, n)
    out.lam = rays["lam"].cpu().numpy()
    out.attempts = rays["attempts"].cpu().numpy().view(np.uint32)
    out.accepted = rays["accepted"].cpu().numpy().view(np.uint32)
    out.intensity = rays["intensity"].cpu().numpy()
    out.color_temp = rays["color_temp"].cpu().numpy()
    out.rgb = rays["rgb"].cpu().numpy().reshape(n, 3)
    out.cross = rays["cross"].cpu().numpy().reshape(8, n)
    return img, out


def same(a: RayOutputs, b: RayOutputs) -> None:
    # same kernels on the same inputs: identical, which is within the 1e-9
    # endpoint tolerance of the parity tests
    for f in FIELDS:
        x, y = getattr(a, f), getattr(b, f)
        assert np.array_equal(x, y, equal_nan=True), f


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    torch.cuda.init()
    return torch


@pytest.mark.parametrize("supersampled", [True, False], ids=["spa2", "spp1"])
def test_noalloc_matches_context_render_twice(torch_cuda, supersampled):
    scene = workloads.schwarzschild_thin_256()
    if supersampled:
        scene.width = scene.height = 96
        scene.options.samples_per_axis = 2
    r = Renderer(0)
    try:
        want_img, want = r.render(scene, rays=True)
    finally:
        r.close()
    for _ in range(2):
        img, got = noalloc_render(torch_cuda, scene)
        assert np.array_equal(img, want_img)
        same(got, want)


def test_noalloc_kerr_scene_matches(torch_cuda):
    scene = workloads.kerr_thin_1080p()
    scene.width, scene.height = 320, 180
    r = Renderer(0)
    try:
        want_img, want = r.render(scene, rays=True)
    finally:
        r.close()
    img, got = noalloc_render(torch_cuda, scene)
    assert np.array_equal(img, want_img)
    same(got, want)


def test_noalloc_supersampling_at_the_scratch_limit(torch_cuda):
    # 680 x 257 pixels x 4 samples = 699,040, the last sample's colour ending
    # exactly at the end of the array
    scene = workloads.schwarzschild_thin_256()
    scene.width, scene.height = 680, 257
    scene.options.samples_per_axis = 2
    assert scene.n_samples == 699040
    r = Renderer(0)
    try:
        want_img, want = r.render(scene, rays=True)
    finally:
        r.close()
    img, got = noalloc_render(torch_cuda, scene)
    assert np.array_equal(img, want_img)
    same(got, want)


def test_noalloc_second_call_allocates_nothing(torch_cuda):
    # after a first call has loaded the module on this device, a call leaves
    # the device's free memory exactly as it was
    scene = workloads.schwarzschild_thin_256()
    scene.width = scene.height = 64
    scene.options.samples_per_axis = 2
    noalloc_render(torch_cuda, scene)
    lib = abi.load()
    rgb = torch_cuda.zeros(scene.width * scene.height * 3, dtype=torch_cuda.uint8, device="cuda")
    torch_cuda.cuda.synchronize()
    free0, _ = torch_cuda.cuda.mem_get_info()
    st = lib.gg_render_device_noalloc(*scene.c_args(), C.c_void_p(rgb.data_ptr()), None, None)
    torch_cuda.cuda.synchronize()
    free1, _ = torch_cuda.cuda.mem_get_info()
    assert st == abi.GG_OK
    assert free1 == free0


@pytest.mark.parametrize("shape", [(1024, 1024, 2, 0), (2699, 37, 1, 7)],
                         ids=["4M-samples", "one-past-the-limit"])
def test_noalloc_rejects_oversized_supersampling(torch_cuda, shape):
    w, h, spa, jitter = shape
    scene = workloads.schwarzschild_thin_256()
    scene.width, scene.height = w, h
    scene.options.samples_per_axis = spa
    scene.options.jitter_spp = jitter
    assert scene.n_samples in (4194304, 699041)
    rgb = torch_cuda.zeros(16, dtype=torch_cuda.uint8, device="cuda")
    lib = abi.load()
    st = lib.gg_render_device_noalloc(*scene.c_args(), C.c_void_p(rgb.data_ptr()), None, None)
    assert st == abi.GG_ERR_TOO_LARGE
    assert b"scratch" in lib.gg_strerror(st)
