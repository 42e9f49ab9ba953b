"""bench.py's multi-rank host logic on two gloo ranks (127.0.0.1): the
barrier, the sum and the max over ranks that make the whole-job value
(units of all ranks over the slowest rank's time), and the per-rank camera
orbit of the frame-per-rank form.  Under torchrun on GPUs the same helpers
run over NCCL with device tensors."""
from __future__ import annotations

import math
import os
import socket

import pytest


def _worker(rank, world, port, q):
    import torch.distributed as dist

    import bench
    from gargantua_b200 import workloads
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        bench.barrier(world)
        total = bench.sum_over_ranks(1000 + rank, world)
        slowest = bench.max_over_ranks(2.5 * (rank + 1), world)
        sc = workloads.kerr_thin_1080p()
        mine = bench.orbit_frame(sc, rank, world)
        t, r, th, ph = mine.camera.position
        q.put((rank, total, slowest, (r, th, ph), tuple(sc.camera.position)))
    finally:
        dist.destroy_process_group()


def test_rank_reductions_and_orbit_on_two_gloo_ranks():
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
    assert all(p.exitcode == 0 for p in procs)
    got = dict((v[0], v[1:]) for v in (q.get(timeout=10) for _ in procs))
    for rank in (0, 1):
        total, slowest, (r, th, ph), orig = got[rank]
        assert total == 1000 + 1001
        assert slowest == 5.0
        assert r == orig[1] and th == orig[2]
        assert ph == pytest.approx(math.pi * rank)


def test_one_rank_helpers_need_no_process_group():
    import bench
    from gargantua_b200 import workloads
    bench.barrier(1)
    assert bench.sum_over_ranks(7, 1) == 7
    assert bench.max_over_ranks(1.25, 1) == 1.25
    sc = workloads.kerr_thin_1080p()
    assert bench.orbit_frame(sc, 0, 1) is sc
