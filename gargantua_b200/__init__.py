"""gargantua_b200: B200-native (sm_100a) general-relativistic ray path of gargantua.

Null geodesics in the Schwarzschild and Kerr metrics are integrated on the GPU
with gargantua's adaptive RK45 (Dormand-Prince) stepper, terminated at the
horizon, the accretion disk or the escape sphere, and shaded.  The compute
runs in ``libgargantua_gpu.so`` (hand-written CUDA behind a C ABI declared in
``include/gargantua_gpu.h``); this package is the host-side mirror of the
reference's ``gr-core`` / ``raytracer::curved`` API over that ABI.
"""
from .gr_core import Kerr, RK45Integrator, Schwarzschild  # noqa: F401
from .curved import (AccretionDisk, Camera, CheckerSky, ProceduralSky, RenderOptions,  # noqa: F401
                     Renderer, Scene, ThinDisk, render, render_with_disk)

__version__ = "0.1.0"
