"""Work split across GPUs (gargantua_b200.shard): a frame by interleaved
rows, a batch by whole scenes.

CPU: the row partition and the assembly, and the gather itself with two
gloo ranks (127.0.0.1); the scene partition's coverage and balance, and that
two gloo ranks derive the same split.  GPU: the shards a rank would render, stitched,
equal the unsplit render byte for byte (each ray's arithmetic does not
depend on which rows share its launch; jitter is keyed by the sample's
index in the whole image).
"""
from __future__ import annotations

import os

import numpy as np
import pytest

from gargantua_b200 import abi, shard, workloads


@pytest.mark.parametrize("height,world", [(8, 2), (7, 2), (5, 3), (2, 4)])
def test_partition_and_assembly(height, world):
    full = np.arange(height * 3 * 3, dtype=np.int64).reshape(height, 3, 3)
    parts = [full[k::world] for k in range(world)]
    assert sum(shard.rows_of(height, k, world) for k in range(world)) == height
    assert [p.shape[0] for p in parts] == [shard.rows_of(height, k, world) for k in range(world)]
    assert np.array_equal(shard.assemble(parts, height), full)


def _gather_worker(rank, world, port, height, q):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        full = np.arange(height * 4 * 3, dtype=np.uint8).reshape(height, 4, 3)
        local = torch.from_numpy(np.ascontiguousarray(full[rank::world]))
        got = shard.gather_rows(local, height, rank, world)
        if rank == 0:
            q.put(bool(np.array_equal(got, full)))
        else:
            q.put(got is None)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("height", [9, 8])
def test_gather_two_gloo_ranks(height):
    import socket

    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gather_worker, args=(r, 2, port, height, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    assert all(q.get(timeout=10) for _ in procs)


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_scene_partition_covers_and_balances(world):
    scenes = workloads.batch_scenes(256, seed=0)
    parts = shard.partition_scenes(scenes, world)
    assert parts == shard.partition_scenes(scenes, world)  # deterministic
    flat = sorted(k for p in parts for k in p)
    assert flat == list(range(len(scenes)))
    loads = [sum(shard.scene_cost(scenes[k]) for k in p) for p in parts]
    # longest-processing-time-first: within one scene's cost of the mean
    biggest = max(shard.scene_cost(s) for s in scenes)
    assert max(loads) - min(loads) <= biggest


def _partition_worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        scenes = workloads.batch_scenes(64, seed=1)
        mine = shard.partition_scenes(scenes, world)[rank]
        got = [None] * world
        dist.all_gather_object(got, mine)
        if rank == 0:
            flat = sorted(k for p in got for k in p)
            q.put(flat == list(range(len(scenes))))
        else:
            q.put(True)
    finally:
        dist.destroy_process_group()


def test_scene_partition_two_gloo_ranks():
    """Every rank derives the same split on its own: together they render
    every scene exactly once."""
    import socket

    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_partition_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    assert all(q.get(timeout=10) for _ in procs)


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["fp64", "mixed", "jitter"])
def test_shards_equal_the_unsplit_render(renderer, form):
    if form == "mixed":
        scene = workloads.kerr_thin_1080p(precision=abi.GG_PREC_MIXED,
                                          stepper=abi.GG_STEPPER_DP45)
        scene.width, scene.height = 192, 108
    elif form == "jitter":
        scene = workloads.kerr_stress_4k(side=48, spp=4)
    else:
        scene = workloads.schwarzschild_thin_256()
    full, _ = renderer.render(scene)
    world = 3
    parts = []
    for k in range(world):
        img, _ = renderer.render(shard.shard_scene(scene, k, world))
        assert img.shape[0] == shard.rows_of(scene.height, k, world)
        parts.append(img)
    assert np.array_equal(shard.assemble(parts, scene.height), full)


def test_orbit_frames_cost_the_same(oracle_mod):
    """bench.py's weak-scaling frames: rank k's camera is rank 0's moved by
    2 pi k / N in azimuth.  The metric and thin disk are axisymmetric, so every
    frame has the same classes and attempt counts (only the sky differs)."""
    import bench
    base = workloads.kerr_thin_1080p()
    base.width, base.height = 64, 36
    frames = [bench.orbit_frame(base, k, 4) for k in range(4)]
    for f in frames:
        t, r, th, ph = f.camera.position
        assert (r, th) == tuple(base.camera.position[1:3])
        la = np.array(f.camera.look_at)
        rhat = np.array([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)])
        assert np.allclose(la, -rhat, atol=1e-15)
    outs = [oracle_mod.render(f)[1] for f in frames[:2]]
    assert np.array_equal(outs[0].cls, outs[1].cls)
    assert np.array_equal(outs[0].attempts, outs[1].attempts)
