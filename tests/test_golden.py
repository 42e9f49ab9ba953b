"""Pins the C++ oracle against the independent pure-Python restatement.

tests/golden/golden_rays.json is produced by tests/golden/make_golden.py (plain
Python doubles, written from the Rust source).  Both restatements follow the
reference's expression order without fused multiply-adds, so they agree to
the last bit; the test allows 1e-12 relative for libm differences.
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
