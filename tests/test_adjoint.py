"""The differentiable render and its hand-written adjoint.

Configuration: Kerr, 512 x 512, target image at (a = 0.7, inclination 60 deg,
r_cam = 40 M, r_in = r_ISCO, q = 3), forward at the target perturbed by
N(0, 5 %) per parameter (seeded), L2 image loss.  The adjoint gradient with
respect to the five parameters must match central finite differences of the
f64 forward (h = 1e-6 relative) to 1e-4 relative.  Pixels whose colour jumps
between the +h and -h renders (a class or sky-cell boundary crossed: the
image is piecewise smooth) are left out of that loss for both.

Data parallel: rank k of N differentiates rows k, k + N, ... of the image;
the forward's rows equal those of the whole image bit for bit, and the
ranks' gradients (one all-reduce of five numbers; two gloo ranks on the CPU)
add up to the whole image's.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

import os

from gargantua_b200 import abi, diff
from gargantua_b200.curved import Camera, CheckerSky, RenderOptions, Scene, ThinDisk
from gargantua_b200.gr_core import Kerr, RK45Integrator


def test_target_and_perturbation_are_seeded():
    t = diff.target_params()
    assert t[0] == 0.7 and abs(t[1] - math.radians(60.0)) < 1e-15 and t[2] == 40.0
    assert abs(t[3] - Kerr(1.0, 0.7).isco()) < 1e-12 and t[4] == 3.0
    a, b = diff.perturbed_params(0), diff.perturbed_params(0)
    assert np.array_equal(a, b) and not np.array_equal(a, t)
    assert np.all(np.abs(a / t - 1.0) < 0.25)


@pytest.mark.parametrize("height,world", [(512, 1), (512, 4), (95, 3), (5, 8)])
def test_row_shards_partition_the_image(height, world):
    s = diff.DiffScene(width=16, height=height)
    shards = [s.shard(k, world) for k in range(world)]
    assert sum(x.rows for x in shards) == height
    rows = sorted(r for x in shards for r in range(x.row_offset, height, x.row_step))
    assert rows == list(range(height))
    assert all(x.width == s.width and x.max_steps == s.max_steps for x in shards)


@pytest.mark.parametrize("rank,world", [(0, 1), (1, 3)])
def test_scene_at_is_the_forward_render(rank, world):
    """DiffScene.scene_at(p) passes the C ABI the same metric, disk,
    integrator, options and camera as the differentiable forward does: the
    bench takes the forward's attempt count and the oracle's baseline from it."""
    import ctypes as C
    s = diff.DiffScene(width=64, height=48).shard(rank, world)
    p = diff.perturbed_params()
    # DiffRenderer() opens a GPU context; its struct builder needs only .scene
    m, d, integ, opts, incl, r_cam = diff.DiffRenderer._structs(
        type("DR", (), {"scene": s})(), p)
    m2, cam2, d2, integ2, opts2 = s.scene_at(p).c_structs()
    for a, b in ((m, m2), (d, d2), (integ, integ2), (opts, opts2)):
        assert C.string_at(C.addressof(a), C.sizeof(a)) == C.string_at(C.addressof(b), C.sizeof(b))
    cam = abi.gg_camera_t()
    abi.check(abi.load().gg_camera_inclined(C.byref(cam), r_cam, incl, s.fov_y,
                                            s.width / s.height), "gg_camera_inclined")
    assert C.string_at(C.addressof(cam), C.sizeof(cam)) == C.string_at(C.addressof(cam2),
                                                                       C.sizeof(cam2))


def _allreduce_worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        part = np.arange(5, dtype=np.float64) * (rank + 1) + 0.25
        q.put((rank, diff.allreduce_grad(part).tolist()))
    finally:
        dist.destroy_process_group()


def test_gradient_allreduce_two_gloo_ranks():
    """Each rank's dL/dp over its rows, summed over the group."""
    import socket

    import torch.multiprocessing as mp
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_allreduce_worker, args=(r, 2, port, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    for pr in procs:
        pr.join(120)
    assert all(pr.exitcode == 0 for pr in procs)
    want = (np.arange(5, dtype=np.float64) * 3 + 0.5).tolist()
    got = dict(q.get(timeout=10) for _ in procs)
    assert got[0] == want and got[1] == want


def test_gradient_allreduce_single_process_is_identity():
    g = np.array([1.5, -2.0, 0.0, 3.25, 1e-9])
    assert np.array_equal(diff.allreduce_grad(g), g)


@pytest.mark.gpu
def test_row_shards_add_up_to_the_whole_gradient(renderer):
    """Rank k of 3 on rows k::3 (95 rows: 32, 32, 31), one after another on
    one context: each shard's image is those rows of the whole image, and
    the shards' gradients sum to the whole image's."""
    import torch
    s = diff.DiffScene(width=96, height=95)
    full = diff.DiffRenderer(s, renderer)
    target = full.render(diff.target_params()).clone()
    p = diff.perturbed_params()
    img = full.render(p).clone()
    dl = (2.0 * (img - target)).contiguous()
    torch.cuda.current_stream().synchronize()
    g_full = full.backward(dl.data_ptr(), torch.cuda.current_stream().cuda_stream)
    world = 3
    g_sum = np.zeros(5)
    for k in range(world):
        dr = diff.DiffRenderer(s.shard(k, world), renderer)
        img_k = dr.render(p)
        assert img_k.shape == (len(range(k, s.height, world)), s.width, 3)
        assert torch.equal(img_k, img[k::world])
        dl_k = dl[k::world].contiguous()
        torch.cuda.current_stream().synchronize()
        g_sum += dr.backward(dl_k.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert np.all(g_full != 0.0)
    # the same per-pixel terms, summed in another order (block partials, atomics)
    assert np.allclose(g_sum, g_full, rtol=1e-9, atol=0.0), (g_sum, g_full)


@pytest.mark.gpu
def test_forward_matches_render(renderer):
    """The differentiable forward is the FP64 full Dormand-Prince render."""
    s = diff.DiffScene(width=96, height=96)
    dr = diff.DiffRenderer(s, renderer)
    p = diff.perturbed_params()
    img = dr.render(p).cpu().numpy().reshape(-1, 3)
    spin, incl, r_cam, r_in, q = p
    scene = Scene(Kerr(1.0, spin), Camera.inclined(r_cam, incl, s.fov_y, 1.0), 96, 96,
                  ThinDisk(r_in, s.r_outer, q),
                  RenderOptions(sky=CheckerSky(18, 36, 0), max_steps=s.max_steps,
                                integrator=RK45Integrator(max_radius=200.0, rtol=1e-8,
                                                          atol=1e-10,
                                                          stepper=abi.GG_STEPPER_DP45)))
    _, g = renderer.render(scene, rays=True)
    assert (g.cls == 2).sum() > 500
    assert np.allclose(img, g.rgb, rtol=0.0, atol=1e-12)


@pytest.mark.gpu
def test_adjoint_matches_central_differences(renderer):
    import torch
    dr = diff.DiffRenderer(diff.DiffScene(), renderer)
    target = dr.render(diff.target_params()).clone()
    p = diff.perturbed_params()
    report = []
    for i in range(5):
        h = 1e-6 * abs(p[i])
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        ip = dr.render(pp).clone()
        im = dr.render(pm).clone()
        keep = ((ip - im).abs().amax(dim=2) < 1e-2).unsqueeze(2).to(torch.float64)
        lp = (((ip - target) ** 2) * keep).sum().item()
        lm = (((im - target) ** 2) * keep).sum().item()
        fd = (lp - lm) / (2.0 * h)
        img = dr.render(p)  # the forward the adjoint runs after
        dl = (2.0 * (img - target) * keep).contiguous()
        torch.cuda.current_stream().synchronize()
        g = dr.backward(dl.data_ptr(), torch.cuda.current_stream().cuda_stream)
        report.append((diff.PARAMS[i], g[i], fd, int((keep == 0).sum().item())))
        assert abs(fd) > 0.0
        assert abs(g[i] - fd) <= 1e-4 * abs(fd), report


@pytest.mark.gpu
def test_autograd_function_gradient(renderer):
    import torch
    dr = diff.DiffRenderer(diff.DiffScene(width=128, height=128), renderer)
    target = dr.render(diff.target_params()).clone()
    p = torch.tensor(diff.perturbed_params(), dtype=torch.float64, requires_grad=True)
    img = diff.kerr_image(p, dr)
    loss = ((img - target) ** 2).sum()
    loss.backward()
    direct = dr.backward((2.0 * (img.detach() - target)).contiguous().data_ptr(),
                         torch.cuda.current_stream().cuda_stream)
    assert np.allclose(p.grad.numpy(), direct, rtol=1e-12, atol=0.0)
    assert np.all(np.isfinite(direct)) and np.any(direct != 0.0)
