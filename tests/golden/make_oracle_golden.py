"""Writes tests/golden/oracle_c1_c2.npz: the CPU oracle's outcomes on the two
parity workloads, for tests that check the CUDA path without running the
oracle, and that pin the oracle itself against later changes.

* C1, Schwarzschild 256 x 256 thin disk (workloads.schwarzschild_thin_256,
  the reference's step): class and attempt count of all 65,536 samples;
  final x, v of a seeded 4,096-sample subset (numpy default_rng(1)).
* C2, Kerr a=0.9 1920 x 1080 thin disk (workloads.kerr_thin_1080p, the
  reference's step): class, attempts and final x, v of a seeded
  4,096-sample subset (default_rng(2)).

Run from the repository root:  python tests/golden/make_oracle_golden.py
(the oracle is built by `make -C oracle`; the result is deterministic).
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

OUT = Path(__file__).resolve().parent / "oracle_c1_c2.npz"
N_SUB = 4096


def main() -> None:
    from gargantua_b200 import workloads
    from oracle import oracle

    oracle.build()
    c1 = workloads.schwarzschild_thin_256()
    _, r1 = oracle.render(c1)
    idx1 = np.sort(np.random.default_rng(1).choice(c1.n_samples, N_SUB, replace=False))
    c2 = workloads.kerr_thin_1080p()
    idx2 = np.sort(np.random.default_rng(2).choice(c2.n_samples, N_SUB, replace=False))
    r2 = oracle.trace_samples(c2, idx2.astype(np.uint64))
    np.savez_compressed(
        OUT,
        c1_cls=r1.cls.astype(np.int8), c1_attempts=r1.attempts.astype(np.uint16),
        c1_idx=idx1.astype(np.int64), c1_x=r1.x[:, idx1], c1_v=r1.v[:, idx1],
        c2_idx=idx2.astype(np.int64), c2_cls=r2.cls.astype(np.int8),
        c2_attempts=r2.attempts.astype(np.uint16), c2_x=r2.x, c2_v=r2.v)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes)")


if __name__ == "__main__":
    main()
