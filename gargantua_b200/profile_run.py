"""Render one named workload a few times, for profilers and quick timings.

    python -m gargantua_b200.profile_run --workload kerr_thin_1080p --precision mixed
    python -m gargantua_b200.profile_run --workload adjoint_512 --repeats 3
    python -m gargantua_b200.profile_run --workload adjoint_512 --side 128 --repeats 2

Prints the device time and statistics of each render.  Under a profiler,
select the trace launch with its kernel name (trace_mixed_kernel,
trace_fp64_kernel).  adjoint_512 renders the differentiable render's target
once, then runs `repeats` gradients (forward with checkpoints, dL/d(image),
backward) of the 512 x 512 five-parameter configuration.
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
    "adjoint_512": None,
}


def run_adjoint(repeats: int, side: int | None = None) -> None:
    import torch

    from . import diff
    r = Renderer(0)
    scene = diff.DiffScene()
    if side:
        scene.width = scene.height = side
    dr = diff.DiffRenderer(scene, r)
    target = dr.render(diff.target_params()).clone()
    p = diff.perturbed_params(0)
    stream = torch.cuda.current_stream()
    for _ in range(repeats):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        img = dr.render(p)
        st = r.stats()
        dl = (2.0 * (img - target)).contiguous()
        g = dr.backward(dl.data_ptr(), stream.cuda_stream)
        e1.record(stream)
        stream.synchronize()
        print(json.dumps({"workload": "adjoint_512", "side": scene.width, "gradient_ms": e0.elapsed_time(e1),
                          "forward_attempts": st.attempts, "gradient": [float(x) for x in g]}),
              flush=True)
    r.close()


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="kerr_thin_1080p")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="mixed")
    ap.add_argument("--stepper", choices=["reference", "dp45"], default=None,
                    help="default: dp45 for mixed, reference for fp64")
    ap.add_argument("--repeats", type=int, default=1)
    ap.add_argument("--side", type=int, default=None,
                    help="kerr_stress_4k, adjoint_512: image side (a smaller case for profilers)")
    ap.add_argument("--spp", type=int, default=None, help="kerr_stress_4k: samples per pixel")
    ap.add_argument("--width", type=int, default=None,
                    help="render the same view at this width (with --height): a smaller case "
                         "of the same kernel for profilers")
    ap.add_argument("--height", type=int, default=None)
    a = ap.parse_args()
    if a.workload == "adjoint_512":
        run_adjoint(a.repeats, a.side)
        return
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
    if a.width and a.height:
        scene.width, scene.height = a.width, a.height
        scene.camera.aspect = a.width / a.height
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
