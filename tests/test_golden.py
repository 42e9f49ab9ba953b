"""Committed golden vectors.

tests/golden/golden_rays.json is produced by tests/golden/make_golden.py (plain
Python doubles, written from the Rust source).  Both restatements follow the
reference's expression order without fused multiply-adds, so they agree to
the last bit; the test allows 1e-12 relative for libm differences.

tests/golden/oracle_c1_c2.npz is produced by tests/golden/make_oracle_golden.py:
the oracle's outcomes on the 256 x 256 Schwarzschild and 1080p Kerr parity
workloads.  The oracle must reproduce it exactly (CPU), and the CUDA path is
held to it (GPU) without running the oracle.
"""
from __future__ import annotations

import json
import math
from pathlib import Path

import numpy as np
import pytest

from gargantua_b200.curved import (AccretionDisk, Camera, CheckerSky, RenderOptions, Scene,
                                   ThinDisk)
from gargantua_b200.gr_core import Kerr, RK45Integrator, Schwarzschild

GOLDEN = Path(__file__).resolve().parent / "golden" / "golden_rays.json"


def scene_of(case) -> Scene:
    kind, m, a = case["metric"]
    metric = Schwarzschild(m) if kind == "schw" else Kerr(m, a)
    cam = case["cam"]
    camera = Camera(tuple(cam["pos"]), tuple(cam["look_at"]), tuple(cam["up"]), cam["fov"],
                    cam["aspect"])
    d = case["disk"]
    disk = None
    if d and d["kind"] == "vol":
        disk = AccretionDisk(d["r_inner"], d["r_outer"], d["scale_height"], d["density_0"])
    elif d and d["kind"] == "thin":
        disk = ThinDisk(d["r_inner"], d["r_outer"], d["q"])
    I = case["integ"]
    integ = RK45Integrator(I["initial_step"], I["min_step"], I["max_step"], I["tolerance"],
                           I["max_radius"], I["horizon_buffer"], I["rtol"], I["atol"])
    sky = CheckerSky(18, 36, case["sky_seed"]) if case["sky"] == "checker" else None
    opts = RenderOptions(sky=sky, max_steps=case["max_steps"], integrator=integ)
    return Scene(metric, camera, case["w"], case["h"], disk, opts)


def close(a, b, rel=1e-12):
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    return np.all(np.abs(a - b) <= rel * np.maximum(1.0, np.abs(b)))


CASES = json.loads(GOLDEN.read_text())


@pytest.mark.parametrize("entry", CASES, ids=[c["case"]["name"] for c in CASES])
def test_oracle_matches_python_restatement(oracle_mod, entry):
    case, rays = entry["case"], entry["rays"]
    scene = scene_of(case)
    idx = np.array([r["py"] * case["w"] + r["px"] for r in rays], np.uint64)
    out = oracle_mod.trace_samples(scene, idx, threads=1)
    for i, r in enumerate(rays):
        assert out.cls[i] == r["cls"], (i, out.cls[i], r["cls"])
        assert out.attempts[i] == r["attempts"]
        assert out.accepted[i] == r["accepted"]
        assert close(out.x[:, i], r["x"]), (i, out.x[:, i], r["x"])
        assert close(out.v[:, i], r["v"]), (i, out.v[:, i], r["v"])
        assert close(out.lam[i], r["lam"])
        assert close(out.intensity[i], r["intensity"])
        assert close(out.rgb[i], r["rgb"])


def test_golden_covers_every_class_and_disk_kind():
    seen = set()
    kinds = set()
    for e in CASES:
        kinds.add((e["case"]["disk"] or {}).get("kind", "none"))
        for r in e["rays"]:
            seen.add(r["cls"])
    assert {0, 1, 2} <= seen
    assert kinds == {"none", "vol", "thin"}
    assert math.isfinite(CASES[0]["rays"][0]["x"][1])


# ---- oracle outcomes on the parity workloads (tests/golden/make_oracle_golden.py) ----
ORACLE_GOLDEN = Path(__file__).resolve().parent / "golden" / "oracle_c1_c2.npz"


class _Rays:
    def __init__(self, x, v, cls):
        self.x, self.v, self.cls = x, v, cls


def _fixture():
    return np.load(ORACLE_GOLDEN)


def test_oracle_reproduces_committed_vectors(oracle_mod):
    """The oracle still gives the committed outcomes bit for bit: all of C1's
    classes and attempt counts, and the endpoints of both seeded subsets."""
    from gargantua_b200 import workloads
    d = _fixture()
    c1 = workloads.schwarzschild_thin_256()
    _, r1 = oracle_mod.render(c1)
    assert np.array_equal(r1.cls, d["c1_cls"]) and np.array_equal(r1.attempts, d["c1_attempts"])
    i1 = d["c1_idx"]
    assert np.array_equal(r1.x[:, i1], d["c1_x"]) and np.array_equal(r1.v[:, i1], d["c1_v"])
    c2 = workloads.kerr_thin_1080p()
    r2 = oracle_mod.trace_samples(c2, d["c2_idx"].astype(np.uint64))
    assert np.array_equal(r2.cls, d["c2_cls"]) and np.array_equal(r2.attempts, d["c2_attempts"])
    assert np.array_equal(r2.x, d["c2_x"]) and np.array_equal(r2.v, d["c2_v"])


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["c1", "c2"])
def test_gpu_against_committed_vectors(renderer, case):
    """The CUDA FP64 path against the committed oracle outcomes, with the bar
    of the oracle parity tests: class on 99.9 % of samples (the rest lie on
    class boundaries), attempt counts on 99.9 %, endpoints within 1e-9 on
    99.9 % of the subset."""
    from gargantua_b200 import workloads
    from parity import REL, endpoint_err
    d = _fixture()
    scene = workloads.schwarzschild_thin_256() if case == "c1" else workloads.kerr_thin_1080p()
    _, g = renderer.render(scene, rays=True)
    idx = d[f"{case}_idx"]
    if case == "c1":
        assert (g.cls == d["c1_cls"]).mean() >= 0.999
        assert (g.attempts == d["c1_attempts"]).mean() >= 0.999
    cls = d[f"{case}_cls"] if case == "c2" else d["c1_cls"][idx]
    att = d["c2_attempts"] if case == "c2" else d["c1_attempts"][idx]
    same = g.cls[idx] == cls
    assert same.mean() >= 0.999
    assert (g.attempts[idx] == att)[same].mean() >= 0.999
    o = _Rays(d[f"{case}_x"], d[f"{case}_v"], cls)
    e = endpoint_err(scene, g.x[:, idx], g.v[:, idx], o)
    assert (e[same] <= REL).mean() >= 0.999, np.quantile(e[same], 0.999)
