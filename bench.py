#!/usr/bin/env python3
"""Kerr 1080p geodesics/s on B200: plain FP64 and mixed FP32/FP64 forms.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: Kerr a = 0.9, 1920x1080, 1 sample per pixel, camera r = 50 M at 75
deg inclination, 60 deg FOV, thin disk r_ISCO-30 M (q = 3), seeded 18x36
checkerboard sky, RK45 with rtol 1e-8 / atol 1e-10, 10,000 step() calls per
ray, escape at r = 200.  A step is one full render of that frame; the scene
is procedural (nothing to load), so "inputs resident" means the parameter
block only.  Between timed steps a 256 MiB buffer is written to flush L2.

One JSON line on rank 0.  ``value`` is whole-job geodesics/s of the mixed
FP32/FP64 form (full Dormand-Prince stepper; rays of the frame traced to
termination per second).  With N ranks the one frame is split by interleaved
rows (rank k traces rows k, k+N, ...; strong scaling), and each step ends
with the all-gather of every rank's RGB8 rows, the only collective; the
step time is the max over ranks.  ``forms`` times the same frame as the plain
FP64 drop-in (the reference's step) and as FP64 with the mixed form's
stepper; ``mixed_over_fp64`` and ``mixed_over_fp64_dp45`` are the ratios,
``endpoint_error`` the mixed form's crossing-state error and class agreement
against the FP64 kernel on every sample.  ``e2e`` is the headline metric
through the public synchronous call ``gg_render`` into pinned host memory
(parameters in, sRGB image out, copies inside the timed region).

``--workload stress`` runs the near-extremal stress configuration instead (Kerr
a = 0.998, 4096 x 4096 x 16 jittered samples, camera r = 15 M at 85 deg, disk
r_ISCO-25 M, 50,000 step() calls): one frame per form and the distribution of
per-ray attempts, as a separate JSON line.

``--workload batch`` renders 2,048 Kerr scenes of uneven size (spin, camera,
inclination, image side 64..512 and disk drawn per scene) in one persistent
launch from a CUDA graph, with the autotuned kernel variant, against the same
scenes rendered one launch each.

``--workload adjoint`` times the differentiable render's gradient: Kerr
512 x 512, L2 image loss, forward with checkpoints and the adjoint to five
parameters (spin, inclination, r_cam, disk r_in, emissivity index), against
the central differences it replaces, on the GPU and through the oracle.

``--workload features`` times the paths beside it on the reference CLI's
800 x 600 render: the volumetric disk, a sky map, the lensed-spheres scene,
and the command line end to end to a PNG file, each against the oracle.

``--impl reference`` times the CPU restatement of the reference's renderer
(the oracle; the Rust reference cannot be built here) on the host cores on
a bounded seeded sample of the same frame.
"""
from __future__ import annotations

import argparse
import copy
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Kerr 1080p geodesics/s, mixed-FP32 vs plain FP64 on B200 at stated endpoint error"
UNIT = "geodesics/s"
# DRAM bytes (read + write) of one launch of the FP32 pass on the Kerr 1080p
# frame: ncu's dram__bytes_read.sum + dram__bytes_write.sum for that launch
# (the second frame of a two-frame launch list, one pass, clocks not locked),
# in the build with FP64 error sums.  They are the 6.2 MB image, the band
# queue and the argument records of the once-per-ray finish and hand-off calls.
MIXED_PASS_DRAM_BYTES = 3_325_440 + 43_624_448
# Renders of this many samples or more run the mixed form's hand-back rounds
# (kHandBackMinRays in gargantua_b200/csrc/gg_capi.cpp).
HAND_BACK_MIN_SAMPLES = 1 << 20
FLUSH_BYTES = 256 << 20


def dist_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def orbit_frame(scene, rank: int, world: int):
    """`scene` with its camera moved by 2 pi rank / world in azimuth (same r
    and inclination, still looking at the hole with +z up)."""
    import copy
    import math
    if world <= 1:
        return scene
    s = copy.copy(scene)
    t, r, th, _ = scene.camera.position
    ph = 2.0 * math.pi * rank / world
    rhat = (math.sin(th) * math.cos(ph), math.sin(th) * math.sin(ph), math.cos(th))
    cam = copy.copy(scene.camera)
    cam.position = (t, r, th, ph)
    cam.look_at = (-rhat[0], -rhat[1], -rhat[2])
    s.camera = cam
    return s


def workload_config(scene, form: str) -> dict:
    integ = scene.integrator_c()
    return {"workload": "kerr_a0.9_1920x1080_thin_disk", "form": form,
            "width": scene.width, "height": scene.height, "spp": scene.spp,
            "spin": scene.metric.spin, "r_cam": scene.camera.position[1],
            "inclination_deg": round(scene.camera.position[2] * 180.0 / 3.141592653589793, 6),
            "disk": [scene.disk.r_inner, scene.disk.r_outer, scene.disk.emissivity_index],
            "rtol": integ.rtol, "atol": integ.atol, "max_steps": integ.max_steps,
            "max_radius": integ.max_radius, "sky": "checkerboard 18x36 seed 0",
            "l2": "256 MiB write between timed steps"}


# ---- clocks ------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        sel = []
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(device_index).uuid)
            sel = ["-i", uuid if uuid.startswith("GPU-") else f"GPU-{uuid}"]
        except Exception:
            sel = []
        self.p = None
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}",
                                       "--format=csv,noheader,nounits", "-lms", "200"] + sel,
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.p = None
        time.sleep(0.3)

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.p.terminate()
        try:
            self.p.wait(5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.seek(0)
        sm, smax, power, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
                power.append(float(parts[3]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        os.unlink(self.f.name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax),
                "power_w_max": max(power), "samples": len(sm), "reasons": sorted(reasons)}


# ---- our arm -------------------------------------------------------------------
def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def _reduce_device() -> str:
    """Where a reduction's tensor lives: the GPU under NCCL, the host under
    gloo (the CPU tests of these helpers)."""
    import torch.distributed as dist
    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def sum_over_ranks(x: int, world: int) -> int:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.int64, device=_reduce_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return int(t.item())


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=_reduce_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def time_form(r, scene, steps, warmup, world, flush, with_clocks, device_index, gather_rows):
    """Device-timed renders of `scene` (this rank's frame, or its rows of the
    one frame) with device-resident outputs; with `gather_rows` each step also
    gathers every rank's RGB8 rows (NCCL all-gather), the split frame's one
    collective."""
    import torch
    rows = scene.rows
    out = torch.empty(scene.width * rows * 3, dtype=torch.uint8, device="cuda")
    gathered = None
    gather_rows = gather_rows and world > 1
    if gather_rows:
        import torch.distributed as dist
        max_rows = (scene.height + world - 1) // world
        pad = torch.zeros(max_rows * scene.width * 3, dtype=torch.uint8, device="cuda")
        gathered = torch.empty(world * pad.numel(), dtype=torch.uint8, device="cuda")

    def gather():
        if gather_rows:
            pad[: out.numel()] = out
            dist.all_gather_into_tensor(gathered, pad)
    # everything (flush, events, renders) on the library context's own stream
    stream = torch.cuda.ExternalStream(r.stream)
    for _ in range(warmup):
        r.render_device(scene, out.data_ptr(), None, r.stream)
    stream.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(steps)]
    barrier(world)
    torch.cuda.synchronize()
    clk = ClockSampler(device_index) if with_clocks else None
    with torch.cuda.stream(stream):
        for _ in range(warmup if gather_rows else 0):
            gather()
        for i in range(steps):
            flush.zero_()
            ev[i][0].record(stream)
            r.render_device(scene, out.data_ptr(), None, r.stream)
            gather()
            ev[i][1].record(stream)
    stream.synchronize()
    torch.cuda.synchronize()
    barrier(world)
    clocks = clk.stop() if clk else None
    ms = [a.elapsed_time(b) for a, b in ev]
    st = r.stats()
    total_ms = max_over_ranks(sum(ms), world)
    return {"ms": ms, "total_ms": total_ms, "stats": st, "clocks": clocks}


def turned_camera(scene, du: float, dv: float):
    """`scene` with its camera turned so that every pixel's direction moves
    by about du (horizontal) and dv (vertical) image-plane units: look_at
    rotated about the camera's up axis by du tan(fov/2) aspect and towards
    its up vector by dv tan(fov/2)."""
    import copy
    import math

    import numpy as np
    cam = scene.camera
    f = np.array(cam.look_at, float)
    f /= np.linalg.norm(f)
    up = np.array(cam.up, float)
    right = np.cross(f, up)
    right /= np.linalg.norm(right)
    up2 = np.cross(right, f)
    t = math.tan(0.5 * cam.fov_y_radians)
    a_u, a_v = du * t * cam.aspect, dv * t
    g = math.cos(a_u) * f + math.sin(a_u) * right
    g = math.cos(a_v) * g + math.sin(a_v) * up2
    s = copy.copy(scene)
    c = copy.copy(cam)
    c.look_at = tuple(float(x) for x in g)
    s.camera = c
    return s


def fp64_amplification(r, scene64, g64, mask, delta: float = 1e-7):
    """Per ray, how much the FP64 kernel amplifies an image-plane
    perturbation of `delta`: the crossing-state change (crossing_geo_err)
    under a camera turned by delta in u, and in v, over delta; the larger of
    the two (inf where the turned ray does not cross)."""
    import numpy as np

    from gargantua_b200.accuracy import crossing_geo_err
    amp = np.zeros(g64.cls.shape[0])
    for du, dv in ((delta, 0.0), (0.0, delta)):
        _, gt = r.render(turned_camera(scene64, du, dv), rays=True)
        ok = mask & np.isfinite(gt.cross[0])
        e = np.full(amp.shape, np.inf)
        e[ok] = crossing_geo_err(gt.cross[:, ok], g64.cross[:, ok]) / delta
        amp = np.maximum(amp, e)
    return amp


def time_e2e(r, scene, steps, warmup, world):
    import numpy as np
    import torch
    host = torch.empty(scene.width * scene.rows * 3, dtype=torch.uint8,
                       pin_memory=True).numpy()
    for _ in range(warmup):
        r.render_into(scene, host)
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(steps):
        r.render_into(scene, host)
    t1 = time.perf_counter()
    barrier(world)
    el = max_over_ranks(t1 - t0, world)
    assert np.any(host)
    return el


def cpu_baseline(scene, target_s: float = 10.0, what: str = "the 1920x1080 frame") -> dict:
    """The oracle (C++ restatement of the reference renderer, rows over all
    host threads) on a seeded subset of `scene`'s samples sized for about
    `target_s` seconds; geodesics/s extrapolated from the subset."""
    import numpy as np
    from oracle import oracle
    rng = np.random.default_rng(0)
    threads = len(os.sched_getaffinity(0))
    probe = np.sort(rng.choice(scene.n_samples, 2048, replace=False)).astype(np.uint64)
    t0 = time.perf_counter()
    oracle.trace_samples(scene, probe, threads=threads)
    rate = 2048 / (time.perf_counter() - t0)
    n = int(min(scene.n_samples, max(4096, rate * target_s)))
    idx = np.sort(rng.choice(scene.n_samples, n, replace=False)).astype(np.uint64)
    t0 = time.perf_counter()
    oracle.trace_samples(scene, idx, threads=threads)
    el = time.perf_counter() - t0
    return {"value": n / el, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{n} seeded rays of {what} (rng seed 0, {100.0 * n / scene.n_samples:.3g} %), "
                      f"{el:.1f} s on {threads} host threads"}


def cpu_baseline_batch(scenes, target_s: float = 10.0) -> dict:
    """The oracle on seeded rays drawn from 16 seeded scenes of a batch, the
    same number from each, sized for about `target_s` seconds."""
    import numpy as np
    from oracle import oracle
    rng = np.random.default_rng(0)
    threads = len(os.sched_getaffinity(0))
    pick = sorted(rng.choice(len(scenes), 16, replace=False).tolist())

    def run(per):
        t0 = time.perf_counter()
        done = 0
        for k in pick:
            sc = scenes[k]
            m = min(per, sc.n_samples)
            idx = np.sort(rng.choice(sc.n_samples, m, replace=False)).astype(np.uint64)
            oracle.trace_samples(sc, idx, threads=threads)
            done += m
        return done, time.perf_counter() - t0

    n0, el0 = run(128)
    per = int(max(128, 128 * target_s / max(el0, 1e-3)))
    n, el = run(per)
    return {"value": n / el, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{n} seeded rays, {per} from each of 16 seeded scenes of the batch "
                      f"(rng seed 0), {el:.1f} s on {threads} host threads"}


def run_ours(args) -> None:
    import numpy as np
    import torch

    from gargantua_b200 import abi, flops, shard, workloads
    from gargantua_b200.accuracy import crossing_geo_err
    from gargantua_b200.curved import Renderer

    rank, _, local = dist_env()
    world = init_dist(local, 600)
    steps, warmup = args.steps, max(3, args.warmup)
    r = Renderer(local)
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    forms = {}
    # fp64: the drop-in (the reference's RK45 step); fp64_dp45: FP64 with the
    # full Dormand-Prince stepper, the method the mixed form runs; mixed: FP32
    # stages with the FP64 controller and FP64 band
    for form, prec, stepper in (("fp64", abi.GG_PREC_FP64, abi.GG_STEPPER_REFERENCE),
                                ("fp64_dp45", abi.GG_PREC_FP64, abi.GG_STEPPER_DP45),
                                ("mixed", abi.GG_PREC_MIXED, abi.GG_STEPPER_DP45)):
        full = workloads.kerr_thin_1080p(precision=prec, stepper=stepper)
        if world > 1 and args.split == "rows":
            # this rank's interleaved rows of the one frame (strong scaling)
            scene = shard.shard_scene(full, rank, world)
        else:
            # this rank's own frame: the camera moved by 2 pi rank / N in
            # azimuth (frames of an orbit; metric and disk are axisymmetric,
            # so every frame costs the same and only the sky differs)
            full = scene = orbit_frame(full, rank, world)
        res = time_form(r, scene, steps, warmup, world, flush, form == "mixed", local,
                        args.split == "rows")
        st = res["stats"]
        mean_ms = statistics.mean(res["ms"])
        attempts = sum_over_ranks(int(st.attempts), world)
        accepted = sum_over_ranks(int(st.accepted), world)
        # samples of the whole job per step: one frame split, or a frame per rank
        job = full.n_samples * (world if args.split == "frames" else 1)
        forms[form] = {
            "geodesics_per_s": job * steps / (res["total_ms"] * 1e-3),
            "ms_per_step": res["total_ms"] / steps,
            "launch_ms_mean": mean_ms,
            "attempts_per_frame": attempts,
            "accepted_per_frame": accepted,
            "attempts_per_s": attempts * steps / (res["total_ms"] * 1e-3),
            "accepted_steps_per_s": accepted * steps / (res["total_ms"] * 1e-3),
            "samples_per_step": job,
            "class_count": [int(x) for x in st.class_count],
            "fp64_band_rays": int(st.fp64_rays), "fp64_band_attempts": int(st.fp64_attempts),
            "clocks": res["clocks"], "scene": scene, "full": full, "stats_attempts": st.attempts,
        }
    head = "mixed"
    H = forms[head]
    scene = H["scene"]

    # roofline of the trace launches: counted FLOPs per attempt of the full
    # Dormand-Prince step x attempts, against the FP32 FMA peak (97 % of the
    # attempts run in FP32; the FP64 band's share is reported beside it)
    fpa = flops.attempt_flops("kerr", scene.integrator_c().rtol, abi.GG_STEPPER_DP45)
    fpa_reduced = flops.reduced_attempt_flops("kerr", scene.integrator_c().rtol,
                                              abi.GG_STEPPER_DP45)
    fp64_peak = r.fma_peak(fp64=True)
    fp32_peak = r.fma_peak(fp64=False)
    peak = fp32_peak
    # this rank's launches (its attempts over its launch time)
    achieved = int(H["stats_attempts"]) * fpa / (H["launch_ms_mean"] * 1e-3)

    # endpoint error of the mixed form against the FP64 kernel of the same
    # method (held to the CPU oracle at 1e-9 by the parity tests): crossing
    # state of every ray that met the escape sphere or the disk plane
    _, g_mx = r.render(scene, rays=True)
    _, g_64 = r.render(forms["fp64_dp45"]["scene"], rays=True)
    both = np.isfinite(g_mx.cross[0]) & np.isfinite(g_64.cross[0])
    err = crossing_geo_err(g_mx.cross[:, both], g_64.cross[:, both])
    eq = np.quantile(err, [0.5, 0.9, 0.99, 0.999, 0.9999, 1.0]).tolist()
    # rays beyond 1e-6: is each one ill-conditioned at FP32 resolution?  The
    # FP64 kernel re-renders the frame with the camera turned by an
    # image-plane step of 1e-7 in u and in v; a ray whose crossing state then
    # moves by more than 3 x 1e-7 (amplification > 3) cannot hold 1e-6 in any
    # FP32 representation of its state
    amp = fp64_amplification(r, forms["fp64_dp45"]["scene"], g_64, both)
    over = err > 1e-6
    explained = over & (amp[both] > 3.0)
    endpoint = {"reference": "FP64 kernel, same stepper, same samples", "rays": int(both.sum()),
                "measure": "max(|dx_cart|/r, |dv_cart|/|v_cart|, |dt|/t, |dv^t|/v^t) at the "
                           "escape-sphere or disk-plane crossing",
                "p50": eq[0], "p90": eq[1], "p99": eq[2], "p99.9": eq[3], "p99.99": eq[4],
                "max": eq[5], "frac_le_1e-6": float((err <= 1e-6).mean()),
                "over_1e-6": int(over.sum()), "over_1e-6_explained": int(explained.sum()),
                "over_1e-6_unexplained": int((over & ~explained).sum()),
                "frac_le_1e-6_or_explained": float(((err <= 1e-6) | explained).mean()),
                "explained_by": "FP64 kernel re-rendered with the camera turned by a 1e-7 "
                                "image-plane step in u and in v: crossing-state change over "
                                "1e-7 above 3",
                "class_agreement": float((g_mx.cls == g_64.cls).mean())}

    # end to end through gg_render (host pinned output)
    e2e_s = time_e2e(r, scene, steps, warmup, world)

    # per-ray attempt distribution (the untimed render above)
    pct = np.percentile(g_mx.attempts, [50, 90, 99, 99.9, 100]).tolist()

    line = {
        "metric": METRIC, "value": H["geodesics_per_s"], "unit": UNIT, "n_gpus": world,
        "steps": steps, "warmup": warmup, "ms_per_step": H["ms_per_step"],
        "higher_is_better": True,
        "scaling": "strong" if (world > 1 and args.split == "rows") else "weak",
        "vs_baseline": None,
        "dtype": "f32+f64",
        "data": "synthetic: procedural Kerr scene, seeded checkerboard sky",
        "config": workload_config(scene, head),
        "clocks": H["clocks"],
        "e2e": {"value": H["samples_per_step"] * steps / e2e_s, "unit": UNIT,
                "h2d_bytes_per_step": abi.load().gg_struct_size(b"launch_params"),
                "d2h_bytes_per_step": scene.width * scene.rows * 3},
        # per step and rank: the mixed kernel and the FP64 band pass; from 2^20
        # samples per render also the round reset, the mixed pass over the rays
        # the band pass hands back and the last FP64 pass
        "gpu_launches": (5 if scene.n_samples >= HAND_BACK_MIN_SAMPLES else 2) * steps,
        "roofline": {"bound": "fp32", "achieved": achieved / 1e12,
                     "peak": peak / 1e12, "unit": "TFLOP/s", "frac": achieved / peak,
                     # DRAM read + write of the FP32 pass, one launch of this frame
                     # (ncu dram__bytes_{read,write}.sum of that launch)
                     "traffic": MIXED_PASS_DRAM_BYTES,
                     "traffic_unit": "bytes per launch of trace_mixed_kernel",
                     "kernel": "trace_mixed_kernel<Kerr, ThinDisk> + FP64 band pass",
                     "flops_per_attempt": fpa,
                     # the formulation the kernels run (closed-form sparse Christoffels)
                     "flops_per_attempt_reduced": fpa_reduced,
                     "achieved_reduced": achieved * fpa_reduced / fpa / 1e12,
                     "frac_reduced": achieved * fpa_reduced / fpa / peak,
                     "peak_source": "measured in this run by gg_measure_fma_peak (FMA chains);"
                                    " MEASURED_PEAKS.json has no FP64/FP32 ALU figure"},
        "forms": {k: {kk: vv for kk, vv in v.items()
                      if kk not in ("scene", "clocks", "full", "stats_attempts")}
                  for k, v in forms.items()},
        "fma_peak_tflops": {"fp64": fp64_peak / 1e12, "fp32": fp32_peak / 1e12},
        "attempts_per_ray_pct": {"p50": pct[0], "p90": pct[1], "p99": pct[2], "p99.9": pct[3],
                                 "max": pct[4]},
    }
    line["config"]["parallelism"] = (
        f"one frame split by interleaved rows over {world} ranks, RGB8 all-gather"
        if (world > 1 and args.split == "rows") else
        f"one 1080p frame per rank ({world}), camera orbit in azimuth, no collective")
    line["endpoint_error"] = endpoint
    line["mixed_over_fp64"] = H["geodesics_per_s"] / forms["fp64"]["geodesics_per_s"]
    line["mixed_over_fp64_dp45"] = H["geodesics_per_s"] / forms["fp64_dp45"]["geodesics_per_s"]
    cpu = rank == 0 and world == 1 and not args.no_cpu_baseline
    if cpu:
        line["cpu_baseline"] = cpu_baseline(forms["fp64"]["scene"])
    if not args.no_configs:
        # the other configurations, each with its own device time, clocks,
        # attempts, roofline fraction and CPU baseline (short runs)
        peaks = {"fp64": fp64_peak, "fp32": fp32_peak}
        k = min(steps, 10)
        line["c1_schwarzschild_256"] = measure_c1(r, steps, warmup, world, local, flush, peaks,
                                                  cpu)
        line["c3_batch_2048"] = measure_batch(r, 2048, 2, 2, world, rank, local, peaks, cpu,
                                              False, 8.0)
        line["c4_adjoint_512"] = measure_adjoint(r, k, 3, world, rank, local, flush, peaks, cpu,
                                                 8.0)
        line["c5_stress_4096x4096x16"] = measure_stress(r, 4096, 16, world, rank, local, peaks,
                                                        cpu, 8.0)
    r.close()
    close_dist(world)
    if rank == 0:
        print(json.dumps(line), flush=True)


# ---- shared by the configuration measurements ----------------------------------------
def init_dist(local: int, timeout_s: int = 300):
    """Process group of a torchrun launch (NCCL), or None on one GPU."""
    import torch
    rank, world, _ = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=timeout_s),
                                device_id=torch.device(f"cuda:{local}"))
    return world


def close_dist(world: int) -> None:
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def roofline_entry(attempts: int, flops_per_attempt: int, seconds: float, peak: float,
                   bound: str, kernel: str) -> dict:
    """Counted FLOPs of `attempts` RK45 attempts over `seconds`, against the
    FMA peak measured in this run."""
    achieved = attempts * flops_per_attempt / seconds
    return {"bound": bound, "achieved": achieved / 1e12, "peak": peak / 1e12,
            "unit": "TFLOP/s", "frac": achieved / peak, "kernel": kernel,
            "flops_per_attempt": flops_per_attempt,
            "peak_source": "measured in this run by gg_measure_fma_peak (FMA chains)"}


# ---- the 256 x 256 Schwarzschild frame (plain FP64) --------------------------------------
def measure_c1(r, steps: int, warmup: int, world: int, local: int, flush, peaks: dict,
               cpu: bool) -> dict:
    """The plain method on the CPU-runnable frame: Schwarzschild M = 1, 256 x 256,
    camera r = 30 M at 80 deg, thin disk 6-20 M, rtol 1e-8 / atol 1e-10, 10,000
    step() calls, the FP64 drop-in (the reference's step).  Each rank renders
    its own copy of the frame (weak scaling); the CPU baseline traces the whole
    frame through the oracle."""
    from gargantua_b200 import abi, flops, workloads
    scene = workloads.schwarzschild_thin_256()
    res = time_form(r, scene, steps, warmup, world, flush, True, local, False)
    st = res["stats"]
    sec = res["total_ms"] * 1e-3 / steps
    attempts = sum_over_ranks(int(st.attempts), world)
    out = {"workload": "schwarzschild_256x256_thin_disk", "form": "fp64 (reference step)",
           "samples_per_step": scene.n_samples * world,
           "ms_per_step": res["total_ms"] / steps,
           "geodesics_per_s": scene.n_samples * world / sec,
           "attempts_per_frame": attempts, "accepted_per_frame":
               sum_over_ranks(int(st.accepted), world),
           "class_count": [int(x) for x in st.class_count], "clocks": res["clocks"],
           "roofline": roofline_entry(int(st.attempts), flops.attempt_flops(
               "schwarzschild", scene.integrator_c().rtol, abi.GG_STEPPER_REFERENCE),
               statistics.mean(res["ms"]) * 1e-3, peaks["fp64"], "fp64",
               "trace_fp64_kernel<Schwarzschild, ThinDisk>")}
    if cpu:
        out["cpu_baseline"] = cpu_baseline(scene, 30.0, "the 256x256 frame")
    return out


# ---- stress configuration ------------------------------------------------------------
def measure_stress(r, side: int, spp: int, world: int, rank: int, local: int, peaks: dict,
                   cpu: bool, cpu_target_s: float = 10.0) -> dict:
    """Near-extremal Kerr a = 0.998, side x side pixels x spp seeded jittered
    samples (4096 x 4096 x 16 by default), camera r = 15 M at 85 deg, disk
    r_ISCO-25 M, 50,000 step() calls per ray: one frame per form (plain FP64,
    FP64 full Dormand-Prince, mixed), timed with CUDA events after a warm-up
    frame of 256 x 256 x 1, with clocks sampled during the frames, and the
    per-ray attempt distribution.  Per-ray outputs stay on the device
    (attempts and class only).  With N ranks each traces its interleaved rows
    of the frame (shard.shard_scene; jitter is keyed by the global sample, so
    the frame is the same); times are the max over ranks, counts and
    histograms sums."""
    import torch

    from gargantua_b200 import abi, flops, shard, workloads

    n = side * side * spp
    rows = shard.rows_of(side, rank, world)
    n_mine = rows * side * spp
    img = torch.empty(max(1, rows) * side * 3, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.ExternalStream(r.stream)
    edges = [0] + [2 ** k for k in range(17)]  # attempts per ray: [0,1), [1,2), [2,4), ...
    forms, cls_of = {}, {}

    def reduce_sum(xs):
        t = torch.tensor(xs, dtype=torch.int64, device="cuda")
        if world > 1:
            import torch.distributed as dist
            dist.all_reduce(t)
        return t.tolist()

    for form, prec, stepper in (("fp64", abi.GG_PREC_FP64, abi.GG_STEPPER_REFERENCE),
                                ("fp64_dp45", abi.GG_PREC_FP64, abi.GG_STEPPER_DP45),
                                ("mixed", abi.GG_PREC_MIXED, abi.GG_STEPPER_DP45)):
        scene = shard.shard_scene(
            workloads.kerr_stress_4k(precision=prec, side=side, spp=spp, stepper=stepper),
            rank, world)
        # warm-up: the same frame cut to one step() call per ray, which sizes the
        # context's per-sample buffers (the mixed form's queues: 2 x 27 GB at
        # full size) outside the timed region; their allocation would otherwise
        # land between the timing events
        warm = copy.copy(scene)
        warm.options = copy.copy(scene.options)
        warm.options.max_steps = 1
        r.render_device(warm, img.data_ptr(), None, r.stream)
        att = torch.empty(n_mine, dtype=torch.int32, device="cuda")
        cls = torch.empty(n_mine, dtype=torch.int32, device="cuda")
        rays = abi.gg_ray_out_t()
        rays.attempts = C.cast(C.c_void_p(att.data_ptr()), C.POINTER(C.c_uint32))
        rays.cls = C.cast(C.c_void_p(cls.data_ptr()), C.POINTER(C.c_int32))
        stream.synchronize()
        barrier(world)
        clk = ClockSampler(local)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r.render_device(scene, img.data_ptr(), rays, r.stream)
        e1.record(stream)
        stream.synchronize()
        clocks = clk.stop()
        ms = max_over_ranks(e0.elapsed_time(e1), world)
        st = r.stats()
        a = att.to(torch.int64)
        hist = [int(((a >= lo) & (a < hi)).sum()) for lo, hi in zip(edges[:-1], edges[1:])]
        hist.append(int((a >= edges[-1]).sum()))
        sums = reduce_sum([int(st.attempts), int(st.accepted), int(st.fp64_rays),
                           int(st.fp64_attempts)] + [int(x) for x in st.class_count] + hist)
        nc = len(st.class_count)
        mixed = form == "mixed"
        fpa = flops.attempt_flops("kerr", 1e-8, abi.GG_STEPPER_REFERENCE if form == "fp64"
                                  else abi.GG_STEPPER_DP45)
        entry = {"ms": ms, "geodesics_per_s": n / (ms * 1e-3),
                 "attempts": sums[0], "accepted": sums[1],
                 "attempts_per_s": sums[0] / (ms * 1e-3),
                 "class_count": sums[4:4 + nc],
                 "fp64_band_rays": sums[2], "fp64_band_attempts": sums[3],
                 "clocks": clocks,
                 "roofline": roofline_entry(sums[0] // world, fpa, ms * 1e-3,
                                            peaks["fp32" if mixed else "fp64"],
                                            "fp32" if mixed else "fp64",
                                            "trace_mixed_kernel + FP64 band passes" if mixed
                                            else "trace_fp64_kernel<Kerr, ThinDisk>"),
                 "attempts_histogram": {"bin_lower_edges": edges[:-1] + [edges[-1]],
                                        "counts": sums[4 + nc:]}}
        if world == 1:
            q = torch.quantile(a[:: max(1, n // 4_000_000)].double(),
                               torch.tensor([0.5, 0.9, 0.99, 0.999], dtype=torch.float64,
                                            device="cuda")).tolist()
            entry["attempts_per_ray"] = {"p50": q[0], "p90": q[1], "p99": q[2], "p99.9": q[3],
                                         "max": int(a.max())}
        forms[form] = entry
        cls_of[form] = cls
        del att
    agree = reduce_sum([int((cls_of["mixed"] == cls_of["fp64_dp45"]).sum())])[0]
    line = {"metric": "Kerr a=0.998 4096^2 x16 spp stress: geodesics/s and per-ray steps",
            "unit": UNIT, "n_gpus": world, "higher_is_better": True, "scaling": "strong",
            "config": {"workload": f"kerr_a0.998_{side}x{side}x{spp}spp_thin_disk",
                       "r_cam": 15.0, "inclination_deg": 85.0, "disk": "r_ISCO-25M",
                       "max_steps": 50000, "rtol": 1e-8, "atol": 1e-10, "samples": n,
                       "parallelism": f"interleaved rows over {world} rank(s)"},
            "forms": forms,
            "mixed_over_fp64": forms["mixed"]["geodesics_per_s"] / forms["fp64"]["geodesics_per_s"],
            "mixed_over_fp64_dp45": (forms["mixed"]["geodesics_per_s"]
                                     / forms["fp64_dp45"]["geodesics_per_s"]),
            "class_agreement_mixed_vs_fp64_dp45": agree / n}
    if cpu and rank == 0 and world == 1:
        line["cpu_baseline"] = cpu_baseline(workloads.kerr_stress_4k(side=side, spp=spp),
                                            cpu_target_s, f"the {side}x{side}x{spp} spp frame")
    return line


def run_stress(args) -> None:
    """--workload stress: the stress configuration as its own JSON line."""
    from gargantua_b200.curved import Renderer
    rank, _, local = dist_env()
    world = init_dist(local, 600)
    r = Renderer(local)
    peaks = {"fp64": r.fma_peak(fp64=True), "fp32": r.fma_peak(fp64=False)}
    line = measure_stress(r, args.side, args.spp, world, rank, local, peaks,
                          not args.no_cpu_baseline)
    r.close()
    close_dist(world)
    if rank == 0:
        print(json.dumps(line), flush=True)


# ---- batched scenes --------------------------------------------------------------------
def measure_batch(r, n_scenes: int, steps: int, warmup: int, world: int, rank: int,
                  local: int, peaks: dict, cpu: bool, one_launch_each: bool,
                  cpu_target_s: float = 10.0) -> dict:
    """n_scenes independent Kerr scenes of uneven size (workloads.batch_scenes:
    spin, camera distance and inclination, image side 64..512, disk outer
    radius drawn per scene, seed 0), mixed precision, in one persistent
    launch replayed from a CUDA graph, after autotuning the kernel variant on
    every 8th scene.  With N ranks each renders the scenes
    shard.partition_scenes gives it (cost-balanced, no data-path
    collective); a step is timed as the max over ranks.  With
    one_launch_each (N = 1) the same scenes are also rendered one launch
    each."""
    import torch

    from gargantua_b200 import abi, flops, shard, workloads

    scenes = workloads.batch_scenes(n_scenes, seed=0)
    parts = shard.partition_scenes(scenes, world)
    mine = [scenes[k] for k in parts[rank]]
    n = sum(sc.n_samples for sc in scenes)
    pix = sum(sc.width * sc.height for sc in mine)
    out = torch.empty(3 * pix, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.ExternalStream(r.stream)
    t0 = time.perf_counter()
    variant, tune_ms = r.batch_autotune(mine[::8])
    tune_s = time.perf_counter() - t0
    for _ in range(warmup):
        r.render_batch_device(mine, out.data_ptr(), r.stream)
    stream.synchronize()
    ms = []
    barrier(world)
    clk = ClockSampler(local)
    for _ in range(steps):
        barrier(world)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r.render_batch_device(mine, out.data_ptr(), r.stream)
        e1.record(stream)
        stream.synchronize()
        ms.append(max_over_ranks(e0.elapsed_time(e1), world))
    clocks = clk.stop()
    st = r.stats()
    attempts = sum_over_ranks(int(st.attempts), world)
    band_rays = sum_over_ranks(int(st.fp64_rays), world)
    band_att = sum_over_ranks(int(st.fp64_attempts), world)
    rays = sum_over_ranks(int(st.rays), world)
    best = min(ms)
    line = {"metric": "batched scenes: geodesics/s, 2,048 Kerr scenes of uneven size, mixed",
            "unit": UNIT, "n_gpus": world, "higher_is_better": True, "steps": steps,
            "warmup": warmup, "scaling": "strong",
            "config": {"workload": f"batch_{len(scenes)}_kerr_scenes_seed0", "scenes": len(scenes),
                       "samples": n, "sides": "64..512 step 64", "spin": "U[0,0.998]",
                       "r_cam": "U[10,100]", "inclination_deg": "U[5,89]", "r_out": "U[15,40]",
                       "max_steps": 20000,
                       "parallelism": f"scenes over {world} rank(s), cost-balanced "
                                      "(shard.partition_scenes)",
                       "l2": "outputs (3 B per sample, 625 MB) larger than L2"},
            "value": n / (best * 1e-3), "ms_per_batch": ms, "clocks": clocks,
            "rays": rays, "attempts": attempts, "attempts_per_s": attempts / (best * 1e-3),
            "fp64_band_rays": band_rays, "fp64_band_attempts": band_att,
            "roofline": roofline_entry(int(st.attempts), flops.attempt_flops(
                "kerr", 1e-8, abi.GG_STEPPER_DP45), best * 1e-3, peaks["fp32"], "fp32",
                "trace_mixed_kernel<Kerr, ThinDisk, BATCH> + FP64 band passes"),
            "autotune": {"variant": variant, "variant_ms_on_every_8th_scene": tune_ms,
                         "variants": abi.batch_variant_names(),
                         "wall_s": tune_s}}
    if world == 1:
        line["class_count"] = [int(x) for x in st.class_count]
    else:
        line["samples_per_rank"] = [sum(scenes[k].n_samples for k in p) for p in parts]
    if one_launch_each and world == 1:
        # the same scenes, one launch each (single-scene entry point, same kernel family)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        off = 0
        for sc in scenes[:8]:  # warm the single-scene path
            r.render_device(sc, out.data_ptr(), None, r.stream)
        stream.synchronize()
        e0.record(stream)
        for sc in scenes:
            r.render_device(sc, out.data_ptr() + off, None, r.stream)
            off += 3 * sc.width * sc.height
        e1.record(stream)
        stream.synchronize()
        single_ms = e0.elapsed_time(e1)
        line["one_launch_per_scene"] = {"ms": single_ms,
                                        "geodesics_per_s": n / (single_ms * 1e-3)}
        line["batch_over_one_launch_per_scene"] = single_ms / best
    if cpu and rank == 0 and world == 1:
        line["cpu_baseline"] = cpu_baseline_batch(scenes, cpu_target_s)
    return line


def run_batch(args) -> None:
    """--workload batch: the batching configuration as its own JSON line."""
    from gargantua_b200.curved import Renderer
    rank, _, local = dist_env()
    world = init_dist(local)
    r = Renderer(local)
    peaks = {"fp64": r.fma_peak(fp64=True), "fp32": r.fma_peak(fp64=False)}
    line = measure_batch(r, args.scenes, max(1, args.steps // 3), max(3, args.warmup), world,
                         rank, local, peaks, not args.no_cpu_baseline, True)
    r.close()
    close_dist(world)
    if rank == 0:
        print(json.dumps(line), flush=True)


# ---- differentiable render ----------------------------------------------------------
def cpu_baseline_fd(dscene, p, target_s: float = 20.0) -> dict:
    """The central differences the adjoint replaces (ten forwards, h = 1e-6
    relative per parameter) through the oracle on the host cores: each of the
    ten parameter points traced on the same seeded rays of the image, sized
    for about `target_s` seconds in all, extrapolated to the whole image;
    gradients/s."""
    import numpy as np
    from oracle import oracle
    rng = np.random.default_rng(0)
    threads = len(os.sched_getaffinity(0))
    n_img = dscene.width * dscene.height
    points = []
    for i in range(5):
        h = 1e-6 * abs(p[i])
        for sgn in (1.0, -1.0):
            q = np.array(p, dtype=np.float64)
            q[i] += sgn * h
            points.append(dscene.scene_at(q))
    probe = np.sort(rng.choice(n_img, 512, replace=False)).astype(np.uint64)
    t0 = time.perf_counter()
    oracle.trace_samples(points[0], probe, threads=threads)
    per_ray = (time.perf_counter() - t0) / 512
    n = int(min(n_img, max(1024, target_s / 10.0 / per_ray)))
    idx = np.sort(rng.choice(n_img, n, replace=False)).astype(np.uint64)
    el = 0.0
    for sc in points:
        t0 = time.perf_counter()
        oracle.trace_samples(sc, idx, threads=threads)
        el += time.perf_counter() - t0
    fd_s = el * n_img / n
    return {"value": 1.0 / fd_s, "unit": "gradients/s", "cores": threads, "kind": "port",
            "seconds_per_gradient": fd_s,
            "sample": f"{n} seeded rays of the {dscene.width}x{dscene.height} image (rng seed 0) "
                      f"at each of the 10 central-difference points, {el:.1f} s on {threads} "
                      "host threads, extrapolated to the whole image"}


def measure_adjoint(r, steps: int, warmup: int, world: int, rank: int, local: int, flush,
                    peaks: dict, cpu: bool, cpu_target_s: float = 20.0) -> dict:
    """The differentiation configuration: Kerr 512 x 512, L2 loss of the image
    against a target rendered at (a = 0.7, inclination 60 deg, r_cam = 40 M,
    r_in = r_ISCO, q = 3), parameters perturbed by N(0, 5 %) (seed 0).  A step
    is one gradient: the forward with checkpoints every 32 accepted steps
    (gg_forward_ckpt), dL/d(image), and the adjoint (gg_backward) to the five
    parameters.  With N ranks each differentiates its interleaved rows and
    the five sums are all-reduced (NCCL) inside the step, the one
    collective; the step time is the max over ranks.  Beside it at N=1: the
    central differences the adjoint replaces (ten forwards at p +- 1e-6 p_i)
    on the GPU, and through the oracle on the host cores (cpu_baseline)."""
    import numpy as np
    import torch

    from gargantua_b200 import abi, diff, flops

    whole = diff.DiffScene()
    dscene = whole.shard(rank, world)
    dr = diff.DiffRenderer(dscene, r)
    stream = torch.cuda.ExternalStream(r.stream)
    p = diff.perturbed_params(0)
    target = torch.empty(dr.n_values, dtype=torch.float64, device="cuda")
    img = torch.empty_like(target)
    dl = torch.empty_like(target)
    dr.forward_into(diff.target_params(), target.data_ptr(), r.stream)
    stream.synchronize()

    def gradient(ev=None):
        with torch.cuda.stream(stream):
            if ev:
                ev[0].record(stream)
            dr.forward_into(p, img.data_ptr(), r.stream)
            if ev:
                ev[1].record(stream)
            torch.sub(img, target, out=dl)
            dl.mul_(2.0)
            if ev:
                ev[2].record(stream)
            g = dr.backward(dl.data_ptr(), r.stream)
            g = diff.allreduce_grad(g)
            if ev:
                ev[3].record(stream)
        return g

    for _ in range(warmup):
        g = gradient()
    stream.synchronize()
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(steps)]
    barrier(world)
    torch.cuda.synchronize()
    clk = ClockSampler(local)
    for i in range(steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        g = gradient(ev[i])
    stream.synchronize()
    clocks = clk.stop()
    fwd = [e[0].elapsed_time(e[1]) for e in ev]
    bwd = [e[2].elapsed_time(e[3]) for e in ev]
    step_ms = [e[0].elapsed_time(e[3]) for e in ev]
    total_ms = max_over_ranks(sum(step_ms), world)
    fwd_ms = max_over_ranks(statistics.mean(fwd), world)
    bwd_ms = max_over_ranks(statistics.mean(bwd), world)
    ms = total_ms / steps
    n_img = whole.width * whole.height

    # end to end through the torch.autograd.Function (parameters from the
    # host, loss and dL/dp back to the host every step)
    tgt = target.view(dscene.rows, dscene.width, 3)
    e2e_loss = 0.0

    def e2e_step():
        pt = torch.tensor(p, dtype=torch.float64, requires_grad=True)
        out = diff.kerr_image(pt, dr)
        loss = ((out - tgt) ** 2).sum()
        loss.backward()
        gg = diff.allreduce_grad(pt.grad.numpy())
        return float(loss.item()), gg
    for _ in range(warmup):
        e2e_step()
    torch.cuda.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(steps):
        e2e_loss, g_e2e = e2e_step()
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    barrier(world)

    # the forward's FP64 attempts (those of the plain render of the same
    # image), against the FP64 FMA peak
    r.render(dscene.scene_at(p))
    attempts = sum_over_ranks(int(r.stats().attempts), world)
    fpa = flops.attempt_flops("kerr", whole.integrator.rtol, abi.GG_STEPPER_DP45)
    line = {"metric": "Kerr 512^2 adjoint: gradients/s (forward + backward, 5 parameters)",
            "value": steps / (total_ms * 1e-3), "unit": "gradients/s", "n_gpus": world,
            "steps": steps, "warmup": warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: procedural Kerr scene, seeded checkerboard sky",
            "config": {"workload": "kerr_adjoint_512x512_5_params",
                       "target": {"spin": 0.7, "inclination_deg": 60.0, "r_cam": 40.0,
                                  "r_in": "r_ISCO", "emissivity_index": 3.0},
                       "perturbation": "x (1 + N(0, 0.05)), numpy seed 0",
                       "params": list(diff.PARAMS), "loss": "L2 over the linear RGB image",
                       "checkpoint_every_accepted_steps": 32,
                       "max_steps": whole.max_steps, "rtol": whole.integrator.rtol,
                       "atol": whole.integrator.atol,
                       "parallelism": (f"interleaved rows over {world} ranks, all-reduce of the "
                                       "5 gradient sums" if world > 1 else "one GPU"),
                       "l2": "256 MiB write between timed steps"},
            "clocks": clocks,
            "geodesics_per_s": n_img / (ms * 1e-3),
            "forward_ms": fwd_ms, "backward_ms": bwd_ms,
            "gradient": [float(x) for x in g],
            "e2e": {"value": steps / e2e_s, "unit": "gradients/s",
                    "h2d_bytes_per_step": abi.load().gg_struct_size(b"launch_params"),
                    "d2h_bytes_per_step": 5 * 8 + 8,
                    "via": "diff.kerr_image (torch.autograd.Function) + loss.backward()"},
            "gpu_launches": 2 * steps,
            "roofline": dict(roofline_entry(attempts // world, fpa, fwd_ms * 1e-3, peaks["fp64"],
                                            "fp64", "trace_fp64_kernel<Kerr, ThinDisk, DP45, "
                                            "camera, CKPT> (the forward; the backward's "
                                            "stage products are not counted)"),
                             traffic=None, forward_attempts=attempts)}
    if world == 1:
        # central differences on the GPU: ten forwards and their losses, timed
        # on the second of two passes (the first loads the loss's elementwise
        # and reduction kernels, about 80 ms once)
        fd = torch.empty_like(target)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for _ in range(2):
            with torch.cuda.stream(stream):
                e0.record(stream)
                for i in range(5):
                    h = 1e-6 * abs(p[i])
                    for sgn in (1.0, -1.0):
                        q = np.array(p)
                        q[i] += sgn * h
                        dr.forward_into(q, fd.data_ptr(), r.stream)
                        ((fd - target) ** 2).sum()
                e1.record(stream)
            stream.synchronize()
        fd_ms = e0.elapsed_time(e1)
        line["central_differences_gpu"] = {"ms": fd_ms, "adjoint_speedup": fd_ms / ms}
        line["e2e"]["loss"] = e2e_loss
    if cpu and rank == 0 and world == 1:
        line["cpu_baseline"] = cpu_baseline_fd(whole, p, cpu_target_s)
    return line


def run_adjoint(args) -> None:
    """--workload adjoint: the differentiation configuration as its own JSON line."""
    import torch

    from gargantua_b200.curved import Renderer
    rank, _, local = dist_env()
    world = init_dist(local)
    r = Renderer(local)
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    peaks = {"fp64": r.fma_peak(fp64=True), "fp32": r.fma_peak(fp64=False)}
    line = measure_adjoint(r, args.steps, max(3, args.warmup), world, rank, local, flush, peaks,
                           not args.no_cpu_baseline)
    r.close()
    close_dist(world)
    if rank == 0:
        print(json.dumps(line), flush=True)


# ---- the next-tier paths ---------------------------------------------------------------
def feature_scenes():
    """The reference CLI's render (800 x 600, camera r = 30 M on the equator,
    procedural sky, FP64 reference step; crates/gr-renderer/src/main.rs:78-137)
    with each path beside the thin-disk ray path: the volumetric disk, a sky
    map, and the lensed-spheres scene."""
    from gargantua_b200 import workloads
    from gargantua_b200.curved import HdriSky
    cases = {}
    cases["volumetric_disk_schwarzschild"] = workloads.reference_cli(disk=True)
    cases["volumetric_disk_kerr_a0.9"] = workloads.reference_cli(metric="kerr", disk=True)
    sc = workloads.reference_cli(metric="kerr")
    sc.options.sky = HdriSky(workloads.synthetic_sky_map())
    cases["sky_map_kerr_a0.9"] = sc
    sc = workloads.reference_cli()
    sc.objects = workloads.lensed_spheres()
    cases["lensed_spheres_schwarzschild"] = sc
    sc = workloads.reference_cli(metric="kerr", disk=True)
    sc.objects = workloads.lensed_spheres()
    cases["lensed_spheres_volumetric_disk_kerr_a0.9"] = sc
    return cases


def run_features(args) -> None:
    """The paths beside the thin-disk ray path, each timed on the GPU (CUDA
    events, device output) and through the oracle on the host cores (a seeded
    sample of the same render): the reference's volumetric disk, its sky map,
    its scene chords (lensed spheres), and the command line end to end to a
    PNG file (wall clock).  One GPU; under torchrun the other ranks exit."""
    import numpy as np
    import torch

    from gargantua_b200 import cli
    from gargantua_b200.curved import Renderer
    from oracle import oracle

    rank, world, local = dist_env()
    if rank != 0:
        return
    torch.cuda.set_device(local)
    r = Renderer(local)
    stream = torch.cuda.ExternalStream(r.stream)
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    threads = len(os.sched_getaffinity(0))
    steps, warmup = args.steps, max(3, args.warmup)
    rng = np.random.default_rng(0)
    cases, clk_all = {}, []
    for name, sc in feature_scenes().items():
        img = torch.empty(sc.width * sc.height * 3, dtype=torch.uint8, device="cuda")
        for _ in range(warmup):
            r.render_device(sc, img.data_ptr(), None, r.stream)
        stream.synchronize()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(steps)]
        clk = ClockSampler(local)
        with torch.cuda.stream(stream):
            for e0, e1 in ev:
                flush.zero_()
                e0.record(stream)
                r.render_device(sc, img.data_ptr(), None, r.stream)
                e1.record(stream)
        stream.synchronize()
        clk_all.append(clk.stop())
        ms = [a.elapsed_time(b) for a, b in ev]
        st = r.stats()
        n = sc.n_samples
        # the oracle on a seeded sample sized for about 3 s
        probe = np.sort(rng.choice(n, 256, replace=False)).astype(np.uint64)
        t0 = time.perf_counter()
        oracle.trace_samples(sc, probe, threads=threads)
        per = (time.perf_counter() - t0) / 256
        m = int(min(n, max(1024, 3.0 / max(per, 1e-9))))
        idx = np.sort(rng.choice(n, m, replace=False)).astype(np.uint64)
        t0 = time.perf_counter()
        oracle.trace_samples(sc, idx, threads=threads)
        el = time.perf_counter() - t0
        best = statistics.median(ms)
        cases[name] = {"width": sc.width, "height": sc.height, "ms": best,
                       "geodesics_per_s": n / (best * 1e-3),
                       "attempts": int(st.attempts), "class_count": [int(x) for x in st.class_count],
                       "cpu_geodesics_per_s": m / el,
                       "gpu_over_cpu": (n / (best * 1e-3)) / (m / el),
                       "cpu_sample": f"{m} seeded samples, {el:.1f} s on {threads} threads"}
    # the command line end to end: scene, render into host memory, PNG file
    out = Path(tempfile.mkdtemp()) / "cli.png"
    argv = ["--disk", "--quiet", "--output", str(out)]
    import contextlib
    import io
    with contextlib.redirect_stdout(io.StringIO()):  # its "Rendered ..." lines
        for _ in range(warmup):
            assert cli.main(argv, renderer=r) == 0
        t0 = time.perf_counter()
        for _ in range(steps):
            cli.main(argv, renderer=r)
        cli_s = (time.perf_counter() - t0) / steps
    png_bytes = out.stat().st_size
    out.unlink()
    n_cli = 800 * 600
    head = cases["volumetric_disk_schwarzschild"]
    reasons = sorted({x for c in clk_all for x in c.get("reasons", [])})
    line = {"metric": "reference CLI render (800x600) geodesics/s per path: volumetric disk, sky map, "
                      "lensed-spheres scene",
            "value": head["geodesics_per_s"], "unit": UNIT, "n_gpus": 1, "steps": steps,
            "warmup": warmup, "ms_per_step": head["ms"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: procedural scenes, seeded 1024x512 sky map",
            "config": {"workload": "gr_renderer_cli_800x600", "camera": "r=30M, equator, 60 deg FOV",
                       "stepper": "reference RK45 (FP64 drop-in)", "max_steps": 5000,
                       "volumetric_disk": "r 6-20 M, scale height 1 M",
                       "l2": "256 MiB write between timed renders"},
            "clocks": {"per_case": clk_all, "reasons": reasons},
            "cases": cases,
            "cli_png_e2e": {"argv": "gr-renderer --disk (Schwarzschild, 800x600) to a PNG file",
                            "ms": 1e3 * cli_s, "geodesics_per_s": n_cli / cli_s,
                            "png_bytes": png_bytes},
            "gpu_launches": steps * len(cases)}
    r.close()
    print(json.dumps(line), flush=True)


# ---- reference arm ---------------------------------------------------------------
def native_libraries() -> list[str]:
    """Shared objects under this repository mapped into this process."""
    found = set()
    try:
        with open("/proc/self/maps") as f:
            for line in f:
                path = line.split()[-1] if len(line.split()) >= 6 else ""
                if path.endswith(".so") and path.startswith(str(ROOT)):
                    found.add(os.path.relpath(path, ROOT))
    except OSError:
        pass
    return sorted(found)


def run_reference(args) -> None:
    import numpy as np

    from oracle import oracle

    rank, world, _ = dist_env()
    if rank != 0:
        return
    # the scene from the oracle alone: this arm maps none of the product's
    # native code (the line lists what it mapped)
    scene = oracle.kerr_thin_1080p()
    threads = len(os.sched_getaffinity(0))
    rng = np.random.default_rng(0)
    probe = np.sort(rng.choice(scene.n_samples, 2048, replace=False)).astype(np.uint64)
    t0 = time.perf_counter()
    oracle.trace_samples(scene, probe, threads=threads)
    rate = 2048 / (time.perf_counter() - t0)
    steps, warmup = args.steps, max(3, args.warmup)
    per_step_s = args.ref_step_s or min(20.0, 150.0 / (steps + warmup))
    n = int(min(scene.n_samples, max(256, rate * per_step_s)))
    idx = np.sort(rng.choice(scene.n_samples, n, replace=False)).astype(np.uint64)
    for _ in range(warmup):
        oracle.trace_samples(scene, idx[: max(256, n // 8)], threads=threads)
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        oracle.trace_samples(scene, idx, threads=threads)
        times.append(time.perf_counter() - t0)
    value = n * steps / sum(times)
    sample = (f"{n} seeded rays of the 1920x1080 frame per step (rng seed 0) on "
              f"{threads} host threads; C++ f64 restatement of the reference renderer "
              "(the Rust reference cannot be built here)")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
            "n_gpus": world, "steps": steps, "warmup": warmup,
            "ms_per_step": 1e3 * sum(times) / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: procedural Kerr scene, seeded checkerboard sky",
            "config": workload_config(scene, "reference f64 CPU"),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "native_so_loaded": native_libraries()}
    print(json.dumps(line), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-configs", action="store_true",
                    help="kerr1080p: skip the other configurations' entries (256^2 "
                         "Schwarzschild, 2,048-scene batch, 512^2 adjoint, 4096^2 x 16 stress)")
    ap.add_argument("--workload", choices=["kerr1080p", "stress", "batch", "adjoint", "features"],
                    default="kerr1080p",
                    help="stress: the a=0.998 4096^2 x 16 spp configuration (one frame per "
                         "form); batch: 2,048 scenes of uneven size in one launch; adjoint: "
                         "the 512^2 five-parameter gradient; features: the reference CLI render "
                         "with the volumetric disk, a sky map and the lensed-spheres scene")
    ap.add_argument("--scenes", type=int, default=2048, help="batch: number of scenes")
    ap.add_argument("--split", choices=["frames", "rows"], default="frames",
                    help="kerr1080p with N > 1: one frame per rank (weak scaling, no "
                         "collective) or one frame split by rows (strong scaling, an all-gather)")
    ap.add_argument("--ref-step-s", type=float, default=0.0,
                    help="--impl reference: seconds of host work per step (default: the run "
                         "fits in about three minutes)")
    ap.add_argument("--side", type=int, default=4096, help="stress: image side")
    ap.add_argument("--spp", type=int, default=16, help="stress: samples per pixel")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "stress":
        run_stress(args)
    elif args.workload == "batch":
        run_batch(args)
    elif args.workload == "adjoint":
        run_adjoint(args)
    elif args.workload == "features":
        run_features(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
