"""The starfield (ProceduralSky::sample, crates/raytracer/src/curved/sky.rs:26-40)
on identical inputs, bit for bit.

The hash reads the f64 bits of a ray's final direction, so whole-frame
comparisons only show agreement where the GPU's and the oracle's directions
agree.  Here the device hash and the oracle's get the same million
directions (and spatial_dir, tracer.rs:185-189, the same velocities), and a
render's escaped rays are shaded exactly as the oracle's hash shades their
own final velocities.  Integer work: the bar is bit-exact."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from gargantua_b200 import abi, workloads


def special_directions() -> np.ndarray:
    e = [1.0, -1.0, 0.0, -0.0, 1e-300, -1e-300, 5e-324, 0.5, np.sqrt(0.5)]
    g = np.array(np.meshgrid(e, e, e)).reshape(3, -1).T
    return g


def random_directions(n: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return d


def random_velocities(n: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    v = rng.normal(size=(n, 4)) * np.exp(rng.uniform(-20, 20, size=(n, 1)))
    v[: n // 100, 1:] = 0.0  # zero spatial part: spatial_dir's (1, 0, 0)
    return v


def test_batched_oracle_forms_equal_single_ones(oracle_mod):
    d = np.vstack([special_directions(), random_directions(200, 1)])
    rgb = oracle_mod.procedural_sky_n(d)
    v = random_velocities(200, 2)
    dirs = oracle_mod.spatial_dir_n(v)
    for i in range(len(d)):
        one = np.zeros(3)
        oracle_mod.lib().ggo_procedural_sky(oracle_mod._ptr(np.ascontiguousarray(d[i])),
                                            oracle_mod._ptr(one))
        assert np.array_equal(one.view(np.uint64), rgb[i].view(np.uint64))
    for i in range(len(v)):
        one = np.zeros(3)
        oracle_mod.lib().ggo_spatial_dir(oracle_mod._ptr(np.ascontiguousarray(v[i])),
                                         oracle_mod._ptr(one))
        assert np.array_equal(one.view(np.uint64), dirs[i].view(np.uint64))


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    return torch


def device_call(torch, fn, x: np.ndarray, out_cols: int) -> np.ndarray:
    xd = torch.from_numpy(np.ascontiguousarray(x, np.float64)).cuda()
    out = torch.empty((len(x), out_cols), dtype=torch.float64, device="cuda")
    st = fn(C.c_void_p(xd.data_ptr()), C.c_void_p(out.data_ptr()), len(x), None)
    assert st == abi.GG_OK
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.gpu
def test_device_starfield_hash_is_bit_exact(torch_cuda, gglib, oracle_mod):
    d = np.vstack([special_directions(), random_directions(1_000_000, 7)])
    got = device_call(torch_cuda, gglib.gg_check_procedural_sky, d, 3)
    want = oracle_mod.procedural_sky_n(d)
    stars = (want[:, 0] > 0.0).sum()
    assert 4000 < stars < 8000  # 3 in 512 of the directions are stars
    bad = np.nonzero((got.view(np.uint64) != want.view(np.uint64)).any(axis=1))[0]
    assert bad.size == 0, f"{bad.size} directions differ, first {d[bad[:3]]}"


@pytest.mark.gpu
def test_device_spatial_dir_is_bit_exact(torch_cuda, gglib, oracle_mod):
    v = random_velocities(1_000_000, 8)
    got = device_call(torch_cuda, gglib.gg_check_spatial_dir, v, 3)
    want = oracle_mod.spatial_dir_n(v)
    assert np.array_equal(got.view(np.uint64), want.view(np.uint64))


@pytest.mark.gpu
@pytest.mark.parametrize("metric", ["schwarzschild", "kerr"])
def test_escaped_rays_shaded_by_the_oracle_hash_of_their_velocity(renderer, oracle_mod, metric):
    # the reference CLI's view (procedural sky, no disk): every escaped ray's
    # colour is the oracle's starfield at the GPU ray's own final velocity
    scene = workloads.reference_cli(320, 240, metric=metric)
    _, g = renderer.render(scene, rays=True)
    esc = g.cls == abi.GG_CLASS_ESCAPED
    assert esc.sum() > 0.5 * len(g.cls)
    want = oracle_mod.procedural_sky_n(oracle_mod.spatial_dir_n(g.v[:, esc].T))
    assert np.array_equal(g.rgb[esc].view(np.uint64), want.view(np.uint64))
