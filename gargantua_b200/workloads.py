"""Named scenes: the reference's CLI render and the benchmark workloads.

Each function returns a ``Scene`` for one workload by what it is and its
sizes.  The integrator of the disk workloads is the reference's RK45 with
its step bounds and a mixed rtol = 1e-8 / atol = 1e-10 error norm, 10,000
step() calls per ray, escape at r = 200 (renderer.rs:264); `stepper`
selects the reference's step or the full Dormand-Prince method
(abi.GG_STEPPER_DP45), which the precision comparison needs.
"""
from __future__ import annotations

import math

from . import abi
from .curved import (AccretionDisk, Camera, CheckerSky, DiffuseLight, Lambertian, ProceduralSky,
                     RenderOptions, Scene, SceneObjects, Sphere, ThinDisk)
from .gr_core import Kerr, RK45Integrator, Schwarzschild


def disk_integrator(stepper: int = abi.GG_STEPPER_REFERENCE) -> RK45Integrator:
    return RK45Integrator(max_radius=200.0, rtol=1e-8, atol=1e-10, stepper=stepper)


def lensed_spheres() -> SceneObjects:
    """gr-renderer's ``--scene lensed-spheres`` (crates/gr-renderer/src/main.rs:186-215):
    a luminous backdrop sphere behind the hole and four coloured Lambertian
    spheres in a cross, 40-60 M out along the camera's line of sight."""
    return SceneObjects([
        Sphere((-60.0, 0.0, 0.0), 4.0, DiffuseLight((2.0, 1.6, 0.8))),
        Sphere((-40.0, 14.0, 0.0), 3.5, Lambertian((0.85, 0.10, 0.10))),
        Sphere((-40.0, -14.0, 0.0), 3.5, Lambertian((0.10, 0.75, 0.20))),
        Sphere((-40.0, 0.0, 14.0), 3.5, Lambertian((0.15, 0.30, 0.90))),
        Sphere((-40.0, 0.0, -14.0), 3.5, Lambertian((0.95, 0.85, 0.20))),
    ])


def reference_cli(width: int = 800, height: int = 600, metric: str = "schwarzschild",
                  spin: float = 0.9, disk: bool = False, samples: int = 1) -> Scene:
    """gr-renderer's default render (crates/gr-renderer/src/main.rs:78-137):
    camera at r = 30 on the equator looking at the hole, 60 degree FOV,
    procedural sky, optional volumetric disk 6-20 M."""
    m = Schwarzschild(1.0) if metric == "schwarzschild" else Kerr(1.0, spin)
    cam = Camera((0.0, 30.0, math.pi / 2.0, 0.0), (-1.0, 0.0, 0.0), (0.0, 0.0, 1.0),
                 math.radians(60.0), width / height)
    return Scene(m, cam, width, height, AccretionDisk() if disk else None,
                 RenderOptions(samples_per_axis=samples, sky=ProceduralSky()))


def synthetic_sky_map(width: int = 1024, height: int = 512, seed: int = 0):
    """A seeded equirectangular sky map (height, width, 3) float32 linear RGB
    standing in for a Radiance file: a blue gradient from the +z pole to a
    warm horizon band and below it, and 0.2 % of texels as stars of
    brightness 2-20."""
    import numpy as np
    rng = np.random.default_rng(seed)
    th = (np.arange(height, dtype=np.float64) + 0.5) / height * math.pi
    base = np.empty((height, 1, 3))
    base[:, 0, 0] = 0.15 + 0.55 * np.sin(th) ** 4
    base[:, 0, 1] = 0.25 + 0.35 * np.sin(th) ** 2
    base[:, 0, 2] = 0.60 + 0.20 * np.cos(th)
    px = np.repeat(base, width, axis=1)
    stars = rng.random((height, width)) < 0.002
    px[stars] = (2.0 + 18.0 * rng.random((int(stars.sum()), 1))) * np.ones(3)
    return px.astype(np.float32)


def schwarzschild_thin_256(precision: int = abi.GG_PREC_FP64,
                           stepper: int = abi.GG_STEPPER_REFERENCE) -> Scene:
    """Schwarzschild M=1, 256x256, 1 spp, camera r=30 at 80 deg inclination, 60 deg
    FOV, thin disk 6-20 M (q=3), 18x36 checkerboard sky seed 0, all f64."""
    return Scene(Schwarzschild(1.0),
                 Camera.inclined(30.0, math.radians(80.0), math.radians(60.0), 1.0), 256, 256,
                 ThinDisk(6.0, 20.0, 3.0),
                 RenderOptions(sky=CheckerSky(18, 36, 0), max_steps=10000,
                               integrator=disk_integrator(stepper), precision=precision))


def kerr_thin_1080p(spin: float = 0.9, precision: int = abi.GG_PREC_FP64,
                    stepper: int = abi.GG_STEPPER_REFERENCE) -> Scene:
    """Kerr a=0.9, 1920x1080, camera r=50 at 75 deg, disk r_ISCO-30 M (q=3),
    the same checkerboard sky and integrator as the 256x256 Schwarzschild scene."""
    k = Kerr(1.0, spin)
    return Scene(k, Camera.inclined(50.0, math.radians(75.0), math.radians(60.0), 1920 / 1080),
                 1920, 1080, ThinDisk(k.isco(), 30.0, 3.0),
                 RenderOptions(sky=CheckerSky(18, 36, 0), max_steps=10000,
                               integrator=disk_integrator(stepper), precision=precision))


def kerr_stress_4k(precision: int = abi.GG_PREC_FP64, side: int = 4096, spp: int = 16,
                   stepper: int = abi.GG_STEPPER_REFERENCE) -> Scene:
    """Near-extremal Kerr a=0.998, 4096x4096, 16 seeded jittered samples per
    pixel, camera r=15 at 85 deg, disk r_ISCO-25 M, 50,000 step() calls."""
    k = Kerr(1.0, 0.998)
    return Scene(k, Camera.inclined(15.0, math.radians(85.0), math.radians(60.0), 1.0), side,
                 side, ThinDisk(k.isco(), 25.0, 3.0),
                 RenderOptions(sky=CheckerSky(18, 36, 0), jitter_spp=spp, seed=1,
                               max_steps=50000, integrator=disk_integrator(stepper),
                               precision=precision))


def _splitmix64(x: int) -> tuple[int, int]:
    """One SplitMix64 step: (new state, output)."""
    m = (1 << 64) - 1
    x = (x + 0x9E3779B97F4A7C15) & m
    z = x
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & m
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & m
    return x, z ^ (z >> 31)


def batch_scenes(n: int = 2048, seed: int = 0, max_side: int = 512,
                 precision: int = abi.GG_PREC_MIXED) -> list:
    """n independent Kerr scenes of uneven size for one batched render:
    spin a ~ U[0, 0.998], camera r ~ U[10, 100] M, inclination ~ U[5, 89] deg,
    image side ~ U{64, 128, ..., max_side}, thin disk r_ISCO .. r_out with
    r_out ~ U[15, 40] M, sky seed = scene index; SplitMix64 draws from the
    master seed.  All share the full Dormand-Prince integrator (rtol 1e-8,
    atol 1e-10, escape at 200 M) with up to 20,000 step() calls per ray."""
    state = seed
    scenes = []
    sides = max_side // 64

    def uniform():
        nonlocal state
        state, z = _splitmix64(state)
        return (z >> 11) * (1.0 / (1 << 53))

    for k in range(n):
        spin = 0.998 * uniform()
        r_cam = 10.0 + 90.0 * uniform()
        incl = math.radians(5.0 + 84.0 * uniform())
        side = 64 * (1 + min(sides - 1, int(uniform() * sides)))
        r_out = 15.0 + 25.0 * uniform()
        kerr = Kerr(1.0, spin)
        scenes.append(Scene(kerr, Camera.inclined(r_cam, incl, math.radians(60.0), 1.0), side, side,
                            ThinDisk(kerr.isco(), r_out, 3.0),
                            RenderOptions(sky=CheckerSky(18, 36, k), max_steps=20000,
                                          integrator=disk_integrator(abi.GG_STEPPER_DP45),
                                          precision=precision)))
    return scenes
