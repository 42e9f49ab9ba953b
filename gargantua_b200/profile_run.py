"""Render one named workload a few times, for profilers and quick timings.

    python -m gargantua_b200.profile_run --workload kerr_thin_1080p --precision mixed

Prints the device time and statistics of each render.  Under a profiler,
select the trace launch with its kernel name (trace_mixed_kernel,
trace_fp64_kernel).
"""
from __future__ import annotations

import argparse
import json

from . import abi, workloads
from .curved import Renderer

WORKLOADS = {
    "kerr_thin_1080p": workloads.kerr_thin_1080p,
    "schwarzschild_thin_256": workloads.schwarzschild_thin_256,
    "kerr_stress_4k": workloads.kerr_stress_4k,
}


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="kerr_thin_1080p")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="mixed")
    ap.add_argument("--stepper", choices=["reference", "dp45"], default=None,
                    help="default: dp45 for mixed, reference for fp64")
    ap.add_argument("--repeats", type=int, default=1)
    ap.add_argument("--side", type=int, default=None, help="kerr_stress_4k: image side")
    ap.add_argument("--spp", type=int, default=None, help="kerr_stress_4k: samples per pixel")
    a = ap.parse_args()
    prec = abi.GG_PREC_MIXED if a.precision == "mixed" else abi.GG_PREC_FP64
    stepper = a.stepper or ("dp45" if a.precision == "mixed" else "reference")
    kw = {"precision": prec,
          "stepper": abi.GG_STEPPER_DP45 if stepper == "dp45" else abi.GG_STEPPER_REFERENCE}
    if a.workload == "kerr_stress_4k":
        if a.side:
            kw["side"] = a.side
        if a.spp:
            kw["spp"] = a.spp
    scene = WORKLOADS[a.workload](**kw)
    r = Renderer(0)
    for _ in range(a.repeats):
        r.render(scene)
        st = r.stats()
        print(json.dumps({"workload": a.workload, "precision": a.precision, "stepper": stepper,
                          "kernel_ms": st.kernel_ms, "rays": st.rays, "attempts": st.attempts,
                          "accepted": st.accepted, "fp64_rays": st.fp64_rays,
                          "fp64_attempts": st.fp64_attempts}), flush=True)
    r.close()


if __name__ == "__main__":
    main()
