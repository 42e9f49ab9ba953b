"""The mixed FP32/FP64 form (GG_PREC_MIXED, full Dormand-Prince stepper).

Its bar, against the FP64 oracle on the same seeded samples:
  * termination class equal on >= 99.99 % of the frame's samples;
  * crossing state (escape sphere r = max_radius or disk plane, where the
    ray met it) within 1e-6 at the 99th percentile, measured geometrically
    (parity.crossing_geo_err: Cartesian position over r, Cartesian velocity,
    t and dt/dlambda relative) so that angles are not judged against r ~ 200;
  * every ray beyond 1e-6 (but at most 0.05 % of them) one that the FP64
    oracle itself amplifies from an FP32-sized input perturbation by more
    than 3x (parity.fp32_amplification): rays that circle just outside the
    FP64 band are ill-conditioned at FP32 resolution, and no FP32 state can
    hold 1e-6 on them;
and the FP64 band: rays that reach it are finished by the FP64 pass, which
the statistics count.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from gargantua_b200 import abi, workloads
from gargantua_b200.curved import AccretionDisk
from parity import mixed_report


def _mixed(scene_fn, **kw):
    return scene_fn(precision=abi.GG_PREC_MIXED, stepper=abi.GG_STEPPER_DP45, **kw)


# ---- CPU: the polar sincos of the FP32 right-hand side ---------------------------
def test_polar_sincos_within_two_ulp():
    """sincos_polar (the same source the kernel runs) against float64 sin/cos on
    theta in [-pi/4, 5pi/4], the range the mixed stages can reach."""
    lib = abi.load()
    th = np.linspace(-np.pi / 4, 5 * np.pi / 4, 400_001).astype(np.float32)
    s = np.empty_like(th)
    c = np.empty_like(th)
    P = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    assert lib.gg_polar_sincos(P(th), P(s), P(c), C.c_uint32(th.size)) == 0
    t = th.astype(np.float64)
    for got, ref in ((s, np.sin(t)), (c, np.cos(t))):
        ulp = np.spacing(np.abs(ref).astype(np.float32)).astype(np.float64)
        assert (np.abs(got - ref) / ulp).max() <= 2.0


# ---- GPU ------------------------------------------------------------------------
@pytest.mark.gpu
def test_mixed_kerr_1080p_against_oracle_subset(renderer, oracle_mod):
    """16,384 seeded rays of the 1080p frame against the FP64 oracle.  No ray
    beyond 1e-6 is unexplained, and on the explained ones the error stays
    within twice what the oracle itself shows from an FP32-sized (1e-7)
    perturbation of the ray's image-plane point (measured: 0.65 on the
    frame's 804 such rays)."""
    scene = _mixed(workloads.kerr_thin_1080p)
    _, g = renderer.render(scene, rays=True)
    idx = np.sort(np.random.default_rng(7).choice(scene.n_samples, 16384, replace=False))
    ref = workloads.kerr_thin_1080p(stepper=abi.GG_STEPPER_DP45)
    o = oracle_mod.trace_samples(ref, idx.astype(np.uint64))
    oc = oracle_mod.trace_cross(ref, idx.astype(np.uint64))
    assert (g.cls[idx] == o.cls).mean() >= 0.9999
    rep = mixed_report(ref, g.cross[:, idx], oc, oracle_mod, index=idx)
    assert rep["rays"] > 16000
    assert rep["p99"] <= 1e-6 and rep["p99.9"] <= 2e-6, rep
    assert rep["unexplained"] == [], rep
    assert rep["worst_ratio"] <= 2.0, rep
    assert rep["max"] <= 1e-2, rep


@pytest.mark.gpu
def test_mixed_kerr_1080p_classes_and_fp64_band(renderer):
    """Full frame against the FP64 kernel of the same method (itself held to
    the oracle at 1e-9 by test_parity_gpu): class agreement and the FP64 band
    statistics."""
    s64 = workloads.kerr_thin_1080p(stepper=abi.GG_STEPPER_DP45)
    img64, g64 = renderer.render(s64, rays=True)
    scene = _mixed(workloads.kerr_thin_1080p)
    img, g = renderer.render(scene, rays=True)
    st = renderer.stats()
    assert (g.cls == g64.cls).mean() >= 0.9999
    assert st.rays == scene.n_samples and sum(st.class_count) == st.rays
    assert st.attempts == int(g.attempts.sum()) and st.accepted == int(g.accepted.sum())
    # rays that reach the FP64 band are finished in FP64; the band is narrow
    assert 0 < st.fp64_rays < 0.1 * scene.n_samples
    assert 0 < st.fp64_attempts < 0.1 * st.attempts
    close = (np.abs(img.astype(int) - img64.astype(int)) <= 1).all(axis=2)
    assert close.mean() >= 0.999


@pytest.mark.gpu
def test_mixed_schwarzschild_256_against_oracle(renderer, oracle_mod):
    scene = _mixed(workloads.schwarzschild_thin_256)
    _, g = renderer.render(scene, rays=True)
    ref = workloads.schwarzschild_thin_256(stepper=abi.GG_STEPPER_DP45)
    _, o = oracle_mod.render(ref)
    assert (g.cls == o.cls).mean() >= 0.9999
    oc = oracle_mod.trace_cross(ref, np.arange(scene.n_samples, dtype=np.uint64))
    rep = mixed_report(ref, g.cross, oc, oracle_mod)
    assert rep["p99"] <= 1e-6, rep
    assert len(rep["unexplained"]) <= 0.0005 * rep["rays"] + 1, rep


@pytest.mark.gpu
def test_mixed_schwarzschild_1024_with_hand_back(renderer, oracle_mod):
    """From 2^20 samples up the FP64 pass hands rays that leave the band back
    to FP32: the Schwarzschild frame at 1024 x 1024 takes that path and is
    held to the same criteria (seeded 4,096-ray subset against the oracle;
    the full frame's classes against the FP64 kernel)."""
    scene = _mixed(workloads.schwarzschild_thin_256)
    scene.width = scene.height = 1024
    _, g = renderer.render(scene, rays=True)
    st = renderer.stats()
    assert st.fp64_rays > 0 and st.rays == scene.n_samples
    ref = workloads.schwarzschild_thin_256(stepper=abi.GG_STEPPER_DP45)
    ref.width = ref.height = 1024
    _, g64 = renderer.render(ref, rays=True)
    assert (g.cls == g64.cls).mean() >= 0.9999
    idx = np.sort(np.random.default_rng(11).choice(scene.n_samples, 4096, replace=False))
    oc = oracle_mod.trace_cross(ref, idx.astype(np.uint64))
    rep = mixed_report(ref, g.cross[:, idx], oc, oracle_mod, index=idx)
    assert rep["p99"] <= 1e-6, rep
    assert len(rep["unexplained"]) <= 0.0005 * rep["rays"] + 1, rep


@pytest.mark.gpu
def test_mixed_is_reproducible(renderer):
    """Each ray's result does not depend on which rays share its warp: two
    renders of the same frame (dynamic work distribution, so different warp
    compositions) agree bit for bit."""
    scene = _mixed(workloads.kerr_thin_1080p)
    scene.width, scene.height = 640, 360
    _, a = renderer.render(scene, rays=True)
    _, b = renderer.render(scene, rays=True)
    assert np.array_equal(a.cls, b.cls) and np.array_equal(a.attempts, b.attempts)
    assert np.array_equal(a.x, b.x) and np.array_equal(a.v, b.v)
    assert np.array_equal(a.rgb, b.rgb)


@pytest.mark.gpu
def test_mixed_unsupported_combinations(renderer):
    ref_stepper = workloads.kerr_thin_1080p(precision=abi.GG_PREC_MIXED)
    with pytest.raises(abi.GargantuaError) as e:
        renderer.render(ref_stepper)
    assert e.value.status == abi.GG_ERR_UNSUPPORTED
    vol = workloads.reference_cli(32, 24, metric="kerr", disk=True)
    vol.options.precision = abi.GG_PREC_MIXED
    vol.options.integrator = workloads.disk_integrator(abi.GG_STEPPER_DP45)
    assert isinstance(vol.disk, AccretionDisk)
    with pytest.raises(abi.GargantuaError) as e:
        renderer.render(vol)
    assert e.value.status == abi.GG_ERR_UNSUPPORTED


@pytest.mark.gpu
def test_mixed_attempt_budget_stops_promptly(renderer):
    scene = _mixed(workloads.kerr_thin_1080p)
    scene.options.attempt_budget = 100_000
    with pytest.raises(abi.GargantuaError) as e:
        renderer.render(scene)
    assert e.value.status == abi.GG_ERR_BUDGET
    assert renderer.stats().attempts < 50_000_000
    img, _ = renderer.render(_mixed(workloads.schwarzschild_thin_256))
    assert img.shape == (256, 256, 3)
