"""Differentiable Kerr render: gg_forward_ckpt / gg_backward and a
torch.autograd.Function over them.

The image (linear RGB, float64, on the GPU) is a function of five
parameters, in this order:

    p = (spin, inclination, r_cam, disk r_inner, disk emissivity index q)

with the inclined camera (look_at = -r_hat, up = +z), a thin disk and the
full Dormand-Prince stepper in FP64.  ``KerrImage.apply(p, renderer)``
returns the image; ``loss.backward()`` runs the adjoint kernel, which
recomputes each ray's trajectory from checkpoints stored every 32 accepted
steps.  The forward/backward pair keeps its state in the context: run a
backward after its own forward, before the next forward on that context.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import abi
from .curved import CheckerSky, RenderOptions, Renderer, ThinDisk
from .gr_core import Kerr, RK45Integrator

PARAMS = ("spin", "inclination", "r_cam", "r_inner", "emissivity_index")


@dataclass
class DiffScene:
    """Everything of the differentiable render that is not a parameter."""
    width: int = 512
    height: int = 512
    fov_y: float = math.radians(60.0)
    r_outer: float = 20.0
    max_steps: int = 10000
    sky: CheckerSky = field(default_factory=lambda: CheckerSky(18, 36, 0))
    integrator: RK45Integrator = field(default_factory=lambda: RK45Integrator(
        max_radius=200.0, rtol=1e-8, atol=1e-10, stepper=abi.GG_STEPPER_DP45))


class DiffRenderer:
    """A library context running the differentiable render of one DiffScene."""

    def __init__(self, scene: DiffScene | None = None, renderer: Renderer | None = None):
        self.scene = scene or DiffScene()
        self.r = renderer or Renderer(0)
        self._lib = abi.load()

    @property
    def n_values(self) -> int:
        return self.scene.width * self.scene.height * 3

    def _structs(self, p):
        spin, incl, r_cam, r_in, q = (float(x) for x in p)
        m = Kerr(1.0, spin).to_c()
        d = ThinDisk(r_in, self.scene.r_outer, q).to_c()
        integ = self.scene.integrator.to_c(self.scene.max_steps, abi.GG_PREC_FP64)
        opts = RenderOptions(sky=self.scene.sky, max_steps=self.scene.max_steps).to_c()
        return m, d, integ, opts, incl, r_cam

    def forward_into(self, p, rgb_dev: int, stream: int = 0) -> None:
        """Forward pass writing width*height*3 doubles at device address rgb_dev."""
        m, d, integ, opts, incl, r_cam = self._structs(p)
        s = self.scene
        abi.check(self._lib.gg_forward_ckpt(self.r.handle, C.byref(m), r_cam, incl, s.fov_y,
                                            s.width / s.height, C.byref(d), C.byref(integ),
                                            C.byref(opts), s.width, s.height,
                                            C.c_void_p(rgb_dev), C.c_void_p(stream)),
                  "gg_forward_ckpt")

    def backward(self, dl_dev: int, stream: int = 0) -> np.ndarray:
        """dL/dp (5) of the last forward, given dL/d(image) at device address dl_dev."""
        g = (C.c_double * 5)()
        abi.check(self._lib.gg_backward(self.r.handle, C.c_void_p(dl_dev), g, C.c_void_p(stream)),
                  "gg_backward")
        return np.array(list(g))

    def render(self, p):
        """Forward pass into a new torch tensor (height, width, 3), float64, CUDA."""
        import torch
        out = torch.empty(self.n_values, dtype=torch.float64, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream
        self.forward_into(p, out.data_ptr(), stream)
        return out.view(self.scene.height, self.scene.width, 3)


def _autograd_function():
    import torch

    class KerrImage(torch.autograd.Function):
        """image = KerrImage.apply(p, diff_renderer), p a float64 tensor of 5."""

        @staticmethod
        def forward(ctx, p, dr):
            ctx.dr = dr
            return dr.render(p.detach().cpu().tolist())

        @staticmethod
        def backward(ctx, grad_out):
            g = grad_out.contiguous().to(torch.float64)
            stream = torch.cuda.current_stream().cuda_stream
            grad = ctx.dr.backward(g.data_ptr(), stream)
            return torch.tensor(grad, dtype=torch.float64), None

    return KerrImage


_KERR_IMAGE = None


def kerr_image(p, dr: DiffRenderer):
    """Differentiable image of parameters p (torch tensor of 5, float64)."""
    global _KERR_IMAGE
    if _KERR_IMAGE is None:
        _KERR_IMAGE = _autograd_function()
    return _KERR_IMAGE.apply(p, dr)


def target_params() -> np.ndarray:
    """Kerr a = 0.7, inclination 60 deg, r_cam = 40 M, r_in = r_ISCO(0.7), q = 3."""
    return np.array([0.7, math.radians(60.0), 40.0, Kerr(1.0, 0.7).isco(), 3.0])


def perturbed_params(seed: int = 0) -> np.ndarray:
    """The target with each parameter scaled by 1 + N(0, 0.05), seeded."""
    rng = np.random.default_rng(seed)
    return target_params() * (1.0 + 0.05 * rng.standard_normal(5))
