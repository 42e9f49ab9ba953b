"""Work split across GPUs.  One frame: interleaved image rows per rank and
one gather of the RGB8 rows to rank 0.  A batch of scenes: whole scenes per
rank, balanced by their expected cost (``partition_scenes``); rays never
cross ranks, so a batch needs no collective on its data path.

Rank k of N traces rows k, k + N, k + 2N, ... (``RenderOptions.row_offset``
/ ``row_step``): the expensive rays -- the shadow's edge and the photon
ring, in the middle of the frame -- fall on every rank alike, which
contiguous bands would not give.  Rays are independent, so there is no
collective on the data path; the only one is the final gather.  Every rank
calls ``gather_rows`` (same collective, same order); rank 0 returns the
frame.
"""
from __future__ import annotations

import copy

import numpy as np


def rows_of(height: int, rank: int, world: int) -> int:
    """Rows rank `rank` of `world` traces."""
    return 0 if rank >= height else (height - rank + world - 1) // world


def shard_scene(scene, rank: int, world: int):
    """A copy of `scene` that traces this rank's rows."""
    s = copy.copy(scene)
    s.options = copy.copy(scene.options)
    s.options.row_offset = rank
    s.options.row_step = world
    return s


def assemble(parts, height: int):
    """Full image from per-rank row blocks (rank k's block = rows k::N)."""
    world = len(parts)
    width = parts[0].shape[1]
    full = np.zeros((height, width) + tuple(parts[0].shape[2:]), parts[0].dtype)
    for k, part in enumerate(parts):
        full[k::world] = part[: rows_of(height, k, world)]
    return full


def scene_cost(scene) -> float:
    """Expected work of a scene: its samples times the expected attempts per
    ray.  With the step capped at max_step (1 M by default) a ray that
    escapes needs about (its path in and out) / max_step attempts, roughly
    (r_cam + max_radius) / max_step; rays near the hole add a bounded
    share on top."""
    integ = scene.options.integrator
    max_radius = integ.max_radius if integ is not None else 200.0
    max_step = integ.max_step if integ is not None else 1.0
    r_cam = float(scene.camera.position[1])
    return float(scene.n_samples) * (r_cam + max_radius) / max(max_step, 1e-12)


def partition_scenes(scenes, world: int) -> list:
    """Scene indices per rank: longest-processing-time-first greedy on
    scene_cost (each scene to the rank with the least cost so far; ties to
    the lower rank), each rank's list in ascending index order.
    Deterministic, so every rank computes the same split."""
    order = sorted(range(len(scenes)), key=lambda k: (-scene_cost(scenes[k]), k))
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for k in order:
        dst = min(range(world), key=lambda j: (load[j], j))
        parts[dst].append(k)
        load[dst] += scene_cost(scenes[k])
    return [sorted(p) for p in parts]


def gather_rows(local, height: int, rank: int, world: int, group=None):
    """Gathers every rank's rows (torch tensor (rows_k, W, C)) and returns the
    full (height, W, C) image as a numpy array on rank 0, None elsewhere.
    Blocks are padded to the largest share so one all_gather_into_tensor
    moves them (NCCL on GPUs, gloo on the CPU)."""
    import torch
    import torch.distributed as dist
    max_rows = rows_of(height, 0, world)
    pad = torch.zeros((max_rows,) + tuple(local.shape[1:]), dtype=local.dtype,
                      device=local.device)
    pad[: local.shape[0]] = local
    out = torch.empty((world * max_rows,) + tuple(local.shape[1:]), dtype=local.dtype,
                      device=local.device)
    dist.all_gather_into_tensor(out, pad.contiguous(), group=group)
    if rank != 0:
        return None
    blocks = out.view(world, max_rows, *local.shape[1:]).cpu().numpy()
    return assemble([blocks[k] for k in range(world)], height)
