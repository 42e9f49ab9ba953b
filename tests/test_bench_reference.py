"""bench.py's reference arm on the CPU: it times the oracle (the C++
restatement of the reference renderer) on the same frame as the GPU arm, and
maps none of the product's native code while doing so."""
from __future__ import annotations

import ctypes as C
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def test_oracle_scene_equals_the_bench_frame(gglib, oracle_mod):
    from gargantua_b200 import workloads
    a = oracle_mod.kerr_thin_1080p().c_args()
    b = workloads.kerr_thin_1080p().c_args()
    for x, y in zip(a[:5], b[:5]):
        x, y = x._obj, y._obj
        assert type(x) is type(y)
        assert bytes(x) == bytes(y), type(x).__name__
    assert [v.value for v in a[5:]] == [v.value for v in b[5:]] == [1920, 1080]


def test_reference_arm_maps_no_product_library(oracle_mod):
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference",
                          "--steps", "1", "--warmup", "3", "--ref-step-s", "0.05"],
                         capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["value"] > 0 and line["e2e"]["value"] == line["value"]
    assert line["cpu_baseline"]["kind"] == "port"
    assert "oracle/_build/liboracle_gg.so" in line["native_so_loaded"]
    assert not any("libgargantua_gpu" in p for p in line["native_so_loaded"])
    assert line["config"]["workload"] == "kerr_a0.9_1920x1080_thin_disk"
