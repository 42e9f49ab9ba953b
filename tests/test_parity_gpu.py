"""FP64 kernel parity with the CPU oracle, through the C ABI (needs a B200).

Parity bar (plain FP64 form):
  * termination class identical on every sample that is not within 1e-6 M
    (impact parameter) of a class boundary; boundary samples are found by
    re-shooting them on the oracle with the image-plane point moved by that
    margin (oracle.near_class_boundary);
  * final position and velocity (max-norm relative over the four components,
    phi modulo 2 pi; rays ending at the horizon on (r, theta) only, since t,
    phi and the velocity diverge there in Boyer-Lindquist coordinates) within
    1e-9 on 99.9 % of the samples of the 1080p Kerr and 256x256
    Schwarzschild scenes; on every scene the distribution of endpoint
    differences no wider than that of the oracle built with fused
    multiply-adds (the reference algorithm rounded differently), see compare;
  * samples that fail the class test, or a gross-outlier test, must lie
    within 1e-6 M of a class boundary (oracle probe), at most 0.5 % of them;
  * the number of RK45 attempts identical on 99.9 % of agreeing samples;
  * sRGB bytes identical on the checkerboard-sky scenes; with the reference's
    hashed starfield (a hash of the f64 bits of the final direction) the
    background gradient must match and only star placement may differ.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from gargantua_b200 import abi, workloads
from gargantua_b200.curved import CheckerSky, RayOutputs, RenderOptions, Scene, ThinDisk
from gargantua_b200.gr_core import Kerr, Schwarzschild
from parity import compare

pytestmark = pytest.mark.gpu


def test_reference_render_sanity(renderer):
    """render_sanity.rs:16-27 through the GPU: 32x24 has black and non-black pixels."""
    scene = workloads.reference_cli(32, 24)
    img, _ = renderer.render(scene)
    px = img.reshape(-1, 3)
    assert (px == 0).all(axis=1).any()
    assert (px != 0).any(axis=1).any()


def test_schwarzschild_thin_256_full_parity(renderer, oracle_mod):
    scene = workloads.schwarzschild_thin_256()
    img, g = renderer.render(scene, rays=True)
    oimg, o = oracle_mod.render(scene)
    rep = compare(scene, g, o, oracle_mod)
    assert rep["within_1e-9"] > 0.999, rep
    same_px = (img == oimg).all(axis=2)
    assert same_px.mean() > 0.9999, same_px.mean()
    assert np.isin(g.cls, [0, 1, 2]).all()
    assert (g.cls == 2).sum() > 1000 and (g.cls == 0).sum() > 1000


def test_kerr_thin_1080p_seeded_subset(renderer, oracle_mod):
    scene = workloads.kerr_thin_1080p()
    img, g = renderer.render(scene, rays=True)
    rng = np.random.default_rng(0)
    idx = np.sort(rng.choice(scene.n_samples, 4096, replace=False)).astype(np.uint64)
    o = oracle_mod.trace_samples(scene, idx)
    rep = compare(scene, g, o, oracle_mod, idx=idx.astype(np.int64))
    assert rep["within_1e-9"] > 0.999, rep
    # image bytes of the subset's pixels equal the oracle's shading
    lin = o.rgb
    enc = np.clip(lin, 0, 1)
    enc = np.where(enc <= 0.0031308, 12.92 * enc, 1.055 * enc ** (1 / 2.4) - 0.055)
    want = np.rint(enc * 255.0)
    got = img.reshape(-1, 3)[idx.astype(np.int64)]
    assert (np.abs(got - want) <= 1).all(axis=1).mean() > 0.999


def test_reference_cli_procedural_sky(renderer, oracle_mod):
    scene = workloads.reference_cli(160, 120)
    img, g = renderer.render(scene, rays=True)
    oimg, o = oracle_mod.render(scene)
    compare(scene, g, o, oracle_mod)
    # background gradient identical; only hash-placed stars may move
    star_g = (g.rgb[:, 0] > 0) & (g.cls == 1)
    star_o = (o.rgb[:, 0] > 0) & (o.cls == 1)
    plain = ~star_g & ~star_o & (g.cls == o.cls)
    assert np.allclose(g.rgb[plain], o.rgb[plain], rtol=0, atol=1e-9)
    n_esc = (g.cls == 1).sum()
    assert abs(star_g.sum() - star_o.sum()) < max(10, 0.5 * star_o.sum() + 5), \
        (star_g.sum(), star_o.sum(), n_esc)


def test_reference_cli_kerr_volumetric_disk(renderer, oracle_mod):
    scene = workloads.reference_cli(96, 72, metric="kerr", disk=True)
    img, g = renderer.render(scene, rays=True)
    _, o = oracle_mod.render(scene)
    compare(scene, g, o, oracle_mod)
    both_disk = (g.cls == 2) & (o.cls == 2)
    assert both_disk.sum() > 100
    ri = np.abs(g.intensity[both_disk] - o.intensity[both_disk]) / np.abs(o.intensity[both_disk])
    assert np.quantile(ri, 0.999) < 1e-9, ri.max()


def test_supersampling_matches_oracle(renderer, oracle_mod):
    scene = workloads.schwarzschild_thin_256()
    scene.width, scene.height = 64, 64
    scene.options.samples_per_axis = 2
    img, g = renderer.render(scene, rays=True)
    oimg, o = oracle_mod.render(scene)
    compare(scene, g, o, oracle_mod)
    assert (np.abs(img.astype(int) - oimg.astype(int)) <= 1).all(axis=2).mean() > 0.999


def test_jittered_samples_match_oracle(renderer, oracle_mod):
    scene = workloads.kerr_stress_4k(side=48, spp=4)
    scene.options.max_steps = 20000
    img, g = renderer.render(scene, rays=True)
    oimg, o = oracle_mod.render(scene)
    # near-extremal spin seen from r = 15: more photon-ring grazers, whose
    # endpoints diverge chaotically; every other sample must meet 1e-9
    compare(scene, g, o, oracle_mod, max_excluded=0.01)
    assert (np.abs(img.astype(int) - oimg.astype(int)) <= 1).all(axis=2).mean() > 0.99


def test_stress_frame_seeded_subset(renderer, oracle_mod):
    """The full stress frame -- Kerr a = 0.998, 4096 x 4096 x 16 seeded
    jittered samples, camera r = 15 M at 85 deg, 50,000 step() calls -- in
    FP64 on the GPU, and 4,096 seeded samples of it against the oracle.  The
    frame's outputs stay on the device (class, x, v, attempts: 19 GB); only
    the subset comes back."""
    import torch
    scene = workloads.kerr_stress_4k()
    n = scene.n_samples
    assert n == 4096 * 4096 * 16 and scene.options.max_steps == 50000
    cls = torch.empty(n, dtype=torch.int32, device="cuda")
    att = torch.empty(n, dtype=torch.int32, device="cuda")
    x = torch.empty(4 * n, dtype=torch.float64, device="cuda")
    v = torch.empty(4 * n, dtype=torch.float64, device="cuda")
    rays = abi.gg_ray_out_t()
    for name, t, ct in (("cls", cls, C.c_int32), ("attempts", att, C.c_uint32),
                        ("x", x, C.c_double), ("v", v, C.c_double)):
        setattr(rays, name, C.cast(C.c_void_p(t.data_ptr()), C.POINTER(ct)))
    stream = torch.cuda.current_stream(0)
    renderer.render_device(scene, 0, rays, stream.cuda_stream)
    stream.synchronize()
    st = renderer.stats()
    assert st.rays == n
    idx = np.sort(np.random.default_rng(5).choice(n, 4096, replace=False))
    ti = torch.from_numpy(idx.astype(np.int64)).cuda()
    g = RayOutputs(len(idx))
    g.cls = cls[ti].cpu().numpy()
    g.attempts = att[ti].cpu().numpy().view(np.uint32)
    g.x = x.view(4, n)[:, ti].cpu().numpy()
    g.v = v.view(4, n)[:, ti].cpu().numpy()
    del cls, att, x, v
    o = oracle_mod.trace_samples(scene, idx.astype(np.uint64))
    assert o.attempts.max() > 200  # the subset reaches the photon-ring grazers
    compare(scene, g, o, oracle_mod, idx=idx, max_excluded=0.01)


def test_device_pointer_render_matches_host(renderer):
    import torch
    scene = workloads.schwarzschild_thin_256()
    host_img, _ = renderer.render(scene)
    dev = torch.zeros(scene.height * scene.width * 3, dtype=torch.uint8, device="cuda:0")
    stream = torch.cuda.current_stream(0)
    renderer.render_device(scene, dev.data_ptr(), None, stream.cuda_stream)
    stream.synchronize()
    assert np.array_equal(dev.cpu().numpy().reshape(host_img.shape), host_img)
    st = renderer.stats()
    assert st.rays == scene.n_samples and st.attempts >= st.accepted > 0


def test_stats_count_every_ray(renderer):
    scene = workloads.reference_cli(64, 48)
    _, g = renderer.render(scene, rays=True)
    st = renderer.stats()
    assert st.rays == 64 * 48
    assert st.attempts == int(g.attempts.sum())
    assert st.accepted == int(g.accepted.sum())
    assert sum(st.class_count) == st.rays
    assert st.kernel_ms > 0


def test_invalid_arguments_return_status(renderer):
    bad = Scene(Schwarzschild(1.0), workloads.reference_cli(8, 8).camera, 8, 0)
    with pytest.raises(abi.GargantuaError) as e:
        renderer.render(bad)
    assert e.value.status == abi.GG_ERR_INVALID_ARG
    # the context stays usable
    img, _ = renderer.render(workloads.reference_cli(16, 12))
    assert img.shape == (12, 16, 3)


def test_attempt_budget_stops_promptly(renderer):
    scene = workloads.kerr_thin_1080p()
    scene.options.attempt_budget = 100_000
    with pytest.raises(abi.GargantuaError) as e:
        renderer.render(scene)
    assert e.value.status == abi.GG_ERR_BUDGET
    st = renderer.stats()
    assert st.attempts < 50_000_000
    img, _ = renderer.render(workloads.reference_cli(16, 12))
    assert img.shape == (12, 16, 3)


def test_nan_camera_is_rejected_not_traced(renderer):
    s = workloads.reference_cli(8, 8)
    s.camera.position = (0.0, float("nan"), 1.0, 0.0)
    with pytest.raises(abi.GargantuaError):
        renderer.render(s)


def test_thin_disk_every_sample_written(renderer):
    scene = Scene(Kerr(1.0, 0.5), workloads.kerr_thin_1080p().camera, 80, 45,
                  ThinDisk(Kerr(1.0, 0.5).isco(), 30.0, 3.0),
                  RenderOptions(sky=CheckerSky(), max_steps=10000,
                                integrator=workloads.disk_integrator()))
    _, g = renderer.render(scene, rays=True)
    assert np.isin(g.cls, [0, 1, 2, 3]).all()
    esc = g.cls == 1
    assert np.allclose(g.cross[1, esc], 200.0, rtol=1e-12)
    disk = g.cls == 2
    assert np.allclose(g.cross[2, disk], np.pi / 2)
    assert np.isnan(g.cross[:, g.cls == 0]).all()


# ---- full Dormand-Prince stepper (extension) --------------------------------
def test_dp45_schwarzschild_256_full_parity(renderer, oracle_mod):
    scene = workloads.schwarzschild_thin_256(stepper=abi.GG_STEPPER_DP45)
    img, g = renderer.render(scene, rays=True)
    oimg, o = oracle_mod.render(scene)
    rep = compare(scene, g, o, oracle_mod)
    assert rep["within_1e-9"] > 0.999, rep
    assert (img == oimg).all(axis=2).mean() > 0.9999
    assert (g.cls == 2).sum() > 1000


def test_dp45_kerr_1080p_seeded_subset(renderer, oracle_mod):
    scene = workloads.kerr_thin_1080p(stepper=abi.GG_STEPPER_DP45)
    _, g = renderer.render(scene, rays=True)
    idx = np.sort(np.random.default_rng(1).choice(scene.n_samples, 4096, replace=False))
    o = oracle_mod.trace_samples(scene, idx.astype(np.uint64))
    rep = compare(scene, g, o, oracle_mod, idx=idx.astype(np.int64))
    assert rep["within_1e-9"] > 0.999, rep
    # the crossing state (escape sphere / disk plane) from the continuous extension
    oc = oracle_mod.trace_cross(scene, idx.astype(np.uint64))
    gc = g.cross[:, idx]
    m = np.isfinite(oc[0]) & np.isfinite(gc[0])
    assert m.sum() > 3000
    d = np.abs(gc[:, m] - oc[:, m])
    d[3] = np.abs(np.remainder(gc[3, m] - oc[3, m] + np.pi, 2 * np.pi) - np.pi)
    rel = d.max(axis=0) / np.abs(oc[:, m]).max(axis=0)
    assert np.quantile(rel, 0.999) < 1e-9, np.quantile(rel, 0.999)


@pytest.mark.parametrize("w,h", [(1, 1), (1, 37), (33, 1), (7, 5), (31, 3)])
def test_tiny_and_ragged_frames(renderer, oracle_mod, w, h):
    """Frames smaller than one 32-sample chunk or not a multiple of it: every
    sample traced once, classes and endpoints as the oracle's (FP64), classes
    as the FP64 kernel's (mixed form)."""
    scene = workloads.kerr_thin_1080p()
    scene.width, scene.height = w, h
    img, g = renderer.render(scene, rays=True)
    st = renderer.stats()
    assert st.rays == w * h and sum(st.class_count) == w * h and img.shape == (h, w, 3)
    oimg, o = oracle_mod.render(scene)
    assert np.array_equal(g.cls, o.cls) and np.array_equal(g.attempts, o.attempts)
    assert np.array_equal(img, oimg)
    mixed = workloads.kerr_thin_1080p(precision=abi.GG_PREC_MIXED, stepper=abi.GG_STEPPER_DP45)
    ref = workloads.kerr_thin_1080p(stepper=abi.GG_STEPPER_DP45)
    for s in (mixed, ref):
        s.width, s.height = w, h
    imgm, gm = renderer.render(mixed, rays=True)
    assert renderer.stats().rays == w * h
    _, g64 = renderer.render(ref, rays=True)
    assert np.array_equal(gm.cls, g64.cls)


def test_batch_with_tiny_scenes(renderer):
    """A batch whose scenes include 1 x 1 and odd-sized frames: each image as
    the single-scene render's."""
    scenes = workloads.batch_scenes(5, seed=9, max_side=128)
    for s, (w, h) in zip(scenes, [(1, 1), (3, 2), (64, 64), (5, 33), (17, 1)]):
        s.width, s.height = w, h
    imgs = renderer.render_batch(scenes)
    assert renderer.stats().rays == sum(s.n_samples for s in scenes)
    for s, img in zip(scenes, imgs):
        ref, _ = renderer.render(s)
        assert img.shape == (s.height, s.width, 3) and np.array_equal(img, ref)


@pytest.mark.parametrize("stepper", [abi.GG_STEPPER_REFERENCE, abi.GG_STEPPER_DP45],
                         ids=["reference_step", "dp45"])
def test_fp64_is_reproducible(renderer, stepper):
    """A ray's result does not depend on which rays share its warp: two
    renders of a supersampled frame (dynamic work distribution, so different
    warp compositions) agree bit for bit in every output."""
    scene = workloads.schwarzschild_thin_256(stepper=stepper)
    scene.width, scene.height = 680, 257
    scene.options.samples_per_axis = 2
    img_a, a = renderer.render(scene, rays=True)
    img_b, b = renderer.render(scene, rays=True)
    assert np.array_equal(img_a, img_b)
    for f in ("cls", "x", "v", "lam", "attempts", "accepted", "intensity", "color_temp", "rgb",
              "cross"):
        assert np.array_equal(getattr(a, f), getattr(b, f), equal_nan=True), f
