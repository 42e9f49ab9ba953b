"""``python -m gargantua_b200.cli``: the ``gr-renderer`` command line
(crates/gr-renderer/src/main.rs:17-149) on the GPU.

Same arguments, defaults and camera (r = 30 M on the equator looking at the
hole, +z up, 60 degree FOV, aspect width / height), the same dispatch to
``render`` / ``render_with_disk`` (volumetric disk), the optional Radiance
``.hdr`` sky, and a PNG of the frame.  The closing line reads like the
reference's: ``Rendered WxH (metric[+disk]) in T s -> path``, where T runs
from before the sky map is read until the PNG is written.

``--scene lensed-spheres`` (main.rs:186-215) tests every step's chord
against its five spheres on the GPU (render_with_scene, with ``--disk``
render_with_disk_and_scene).

Extensions: ``--precision mixed`` (the FP32/FP64 form, with the full
Dormand-Prince stepper it needs; not with ``--disk`` or a scene),
``--device``.
"""
from __future__ import annotations

import argparse
import math
import sys
import time

from . import abi
from .curved import (AccretionDisk, Camera, HdriSky, ProceduralSky, RenderOptions, Renderer,
                     Scene)
from .gr_core import Kerr, RK45Integrator, Schwarzschild, renderer_integrator
from .png import write_png
from .workloads import lensed_spheres


def parser() -> argparse.ArgumentParser:
    p = argparse.ArgumentParser(prog="gr-renderer", description="General-relativity ray renderer")
    p.add_argument("--metric", default="schwarzschild")
    p.add_argument("--mass", type=float, default=1.0)
    p.add_argument("--spin", type=float, default=0.9)
    p.add_argument("--width", type=int, default=800)
    p.add_argument("--height", type=int, default=600)
    p.add_argument("--disk", action="store_true")
    p.add_argument("--scene", default="none")
    p.add_argument("--r-inner", type=float, default=6.0)
    p.add_argument("--r-outer", type=float, default=20.0)
    p.add_argument("--scale-height", type=float, default=1.0)
    p.add_argument("--samples", type=int, default=1, help="per-axis supersampling")
    p.add_argument("--quiet", action="store_true")
    p.add_argument("--hdri", default=None, help="equirectangular Radiance .hdr sky")
    p.add_argument("--hdri-intensity", type=float, default=1.0)
    p.add_argument("--output", default="out.png")
    p.add_argument("--precision", choices=("fp64", "mixed"), default="fp64")
    p.add_argument("--device", type=int, default=0)
    return p


def build_scene(args) -> Scene:
    """The render main.rs:78-135 sets up, as a Scene."""
    camera = Camera((0.0, 30.0, math.pi / 2.0, 0.0), (-1.0, 0.0, 0.0), (0.0, 0.0, 1.0),
                    math.radians(60.0), args.width / args.height)
    if args.metric == "schwarzschild":
        metric = Schwarzschild(args.mass)
    elif args.metric == "kerr":
        metric = Kerr(args.mass, args.spin)
    else:
        raise ValueError(f"Unknown metric '{args.metric}'. Supported: schwarzschild, kerr")
    if args.scene == "none":
        objects = None
    elif args.scene == "lensed-spheres":
        objects = lensed_spheres()
    else:
        raise ValueError(f"Unknown scene '{args.scene}'. Supported: none, lensed-spheres")
    sky = ProceduralSky()
    if args.hdri is not None:
        try:
            sky = HdriSky.from_file(args.hdri).with_intensity(args.hdri_intensity)
        except (OSError, ValueError) as e:
            raise ValueError(f"failed to load HDRI '{args.hdri}': {e}") from e
    disk = AccretionDisk(r_inner=args.r_inner, r_outer=args.r_outer,
                         scale_height=args.scale_height) if args.disk else None
    opts = RenderOptions(samples_per_axis=max(1, args.samples), show_progress=not args.quiet,
                         sky=sky)
    if args.precision == "mixed":
        base = renderer_integrator()
        opts.integrator = RK45Integrator(max_radius=base.max_radius, rtol=1e-8, atol=1e-10,
                                         stepper=abi.GG_STEPPER_DP45)
        opts.precision = abi.GG_PREC_MIXED
    return Scene(metric, camera, args.width, args.height, disk, opts, objects)


def main(argv=None, renderer: Renderer | None = None) -> int:
    args = parser().parse_args(argv)
    t0 = time.perf_counter()
    try:
        scene = build_scene(args)
    except ValueError as e:
        print(e, file=sys.stderr)
        return 1
    try:
        r = renderer or Renderer(args.device)
        img, _ = r.render(scene)
    except abi.GargantuaError as e:
        print(f"render failed: {e}", file=sys.stderr)
        return 1
    write_png(args.output, img)
    tags = (["disk"] if args.disk else []) + ([args.scene] if args.scene != "none" else [])
    suffix = "+" + "+".join(tags) if tags else ""
    print(f"Rendered {args.width}x{args.height} ({args.metric}{suffix}) in "
          f"{time.perf_counter() - t0:.2f}s → {args.output}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
