"""Builds ``libgargantua_gpu.so`` in-tree for sm_100a with nvcc.

    python -m gargantua_b200.build [--verbose]

``--verbose`` adds ``-Xptxas -v`` (registers, spills and shared memory per
kernel).  Host code is built with ``-ffp-contract=off`` so the per-render
constants it evaluates round exactly like the reference's Rust code.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
import tempfile
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
OUT = PKG / "libgargantua_gpu.so"
SOURCES = ["gg_trace.cu", "gg_mixed.cu", "gg_adjoint.cu", "gg_peak.cu", "gg_capi.cpp",
           "gg_scene_build.cpp", "gg_noalloc.cu", "gg_checks.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise FileNotFoundError("nvcc not found")


def flags(verbose: bool = False) -> list[str]:
    f = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-shared", "--expt-relaxed-constexpr",
                "-Xcompiler", "-fPIC,-fvisibility=hidden,-ffp-contract=off,-O2",
                "-I", str(PKG.parent / "include")]
    if verbose:
        f += ["-Xptxas", "-v"]
    return f


def build(verbose: bool = False, force: bool = False, out: Path | None = None,
          defines: tuple[str, ...] = ()) -> Path:
    """Compiles the library to `out` (default: the in-tree package copy);
    `defines` are extra -D macros (tuning knobs such as GG_TRACE_MIN_BLOCKS)."""
    out = Path(out) if out is not None else OUT
    srcs = [CSRC / s for s in SOURCES]
    deps = srcs + list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + \
        [PKG.parent / "include" / "gargantua_gpu.h"]
    if not force and out.exists() and not verbose and not defines:
        newest = max(p.stat().st_mtime for p in deps)
        if out.stat().st_mtime >= newest:
            return out
    with tempfile.TemporaryDirectory() as tmp:
        tmp_out = Path(tmp) / out.name
        cmd = [nvcc()] + flags(verbose) + [f"-D{d}" for d in defines] + \
            [str(s) for s in srcs] + ["-o", str(tmp_out)]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if verbose or res.returncode != 0:
            sys.stderr.write(res.stdout + res.stderr)
        if res.returncode != 0:
            raise RuntimeError(f"nvcc failed ({res.returncode}): {' '.join(cmd)}")
        out.parent.mkdir(parents=True, exist_ok=True)
        shutil.move(str(tmp_out), out)
    return out


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(a.verbose, a.force))
