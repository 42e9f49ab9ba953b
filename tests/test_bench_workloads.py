"""The inputs bench.py times beside the ray path, on the CPU: the seeded sky
map stands in for a Radiance file, and every case of ``--workload features``
is a render the oracle (its CPU baseline) can trace."""
from __future__ import annotations

import numpy as np
import pytest

import bench
from gargantua_b200 import workloads
from gargantua_b200.curved import AccretionDisk, HdriSky, ProceduralSky


def test_synthetic_sky_map_is_seeded():
    a = workloads.synthetic_sky_map(64, 32, seed=3)
    b = workloads.synthetic_sky_map(64, 32, seed=3)
    c = workloads.synthetic_sky_map(64, 32, seed=4)
    assert a.shape == (32, 64, 3) and a.dtype == np.float32
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    assert np.all(a > 0.0) and np.all(np.isfinite(a))
    big = workloads.synthetic_sky_map()
    assert big.shape == (512, 1024, 3)
    assert 0.001 < (big.max(axis=2) >= 2.0).mean() < 0.004  # the stars


def test_feature_cases():
    cases = bench.feature_scenes()
    assert list(cases) == ["volumetric_disk_schwarzschild", "volumetric_disk_kerr_a0.9",
                           "sky_map_kerr_a0.9", "lensed_spheres_schwarzschild",
                           "lensed_spheres_volumetric_disk_kerr_a0.9"]
    for name, sc in cases.items():
        assert (sc.width, sc.height) == (800, 600), name
        assert isinstance(sc.disk, AccretionDisk) == ("volumetric" in name), name
        assert (sc.objects is not None) == ("lensed" in name), name
        sky = sc.options.sky
        assert isinstance(sky, HdriSky if "sky_map" in name else ProceduralSky), name


@pytest.mark.parametrize("name", list(bench.feature_scenes()))
def test_oracle_traces_each_feature_case(name):
    from oracle import oracle
    sc = bench.feature_scenes()[name]
    idx = np.linspace(0, sc.n_samples - 1, 12).astype(np.uint64)
    ra = oracle.trace_samples(sc, idx, threads=2)
    cls = np.asarray(ra.cls)
    assert np.all((cls >= 0) & (cls <= 5))
    assert np.all(np.asarray(ra.attempts) > 0)


def test_turned_camera_moves_the_view_by_the_image_plane_step():
    # the bench's amplification probe turns the camera so that each pixel
    # moves by about one image-plane step of du (or dv)
    import math
    sc = workloads.kerr_thin_1080p()
    f0 = np.array(sc.camera.look_at) / np.linalg.norm(sc.camera.look_at)
    t = math.tan(0.5 * sc.camera.fov_y_radians)
    for du, dv, want in ((1e-3, 0.0, 1e-3 * t * sc.camera.aspect), (0.0, 1e-3, 1e-3 * t)):
        s2 = bench.turned_camera(sc, du, dv)
        f1 = np.array(s2.camera.look_at)
        assert abs(np.linalg.norm(f1) - 1.0) < 1e-12
        assert abs(math.acos(min(1.0, float(f0 @ f1))) - want) < 1e-9
        assert s2.camera.position == sc.camera.position and s2.camera.up == sc.camera.up
    assert sc.camera.look_at == workloads.kerr_thin_1080p().camera.look_at  # not modified
