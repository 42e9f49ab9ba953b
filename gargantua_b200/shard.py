"""One frame split across GPUs: interleaved image rows per rank and one
gather of the RGB8 rows to rank 0.

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
