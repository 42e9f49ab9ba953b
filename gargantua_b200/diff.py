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

Data parallel over N ranks: ``DiffScene.shard(rank, N)`` traces rows rank,
rank + N, ... (the same interleaving as ``shard.shard_scene``); a loss that
is a sum over pixels then has dL/dp = the sum over ranks of each rank's
backward on its rows, one all-reduce of five numbers (``allreduce_grad``).
"""
from __future__ import annotations

import copy
import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import abi, shard
from .curved import Camera, CheckerSky, RenderOptions, Renderer, Scene, ThinDisk
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
    row_offset: int = 0  # rows traced: row_offset, row_offset + row_step, ...
    row_step: int = 1

    @property
    def rows(self) -> int:
        return shard.rows_of(self.height, self.row_offset, self.row_step)

    def shard(self, rank: int, world: int) -> "DiffScene":
        """A copy tracing rank `rank`'s rows of `world` (interleaved)."""
        s = copy.copy(self)
        s.row_offset, s.row_step = rank, world
        return s

    def scene_at(self, p) -> Scene:
        """The plain render of the same image (same rays, stepper and
        shading) at parameters p, for the render entry points and the oracle."""
        spin, incl, r_cam, r_in, q = (float(x) for x in p)
        return Scene(Kerr(1.0, spin), Camera.inclined(r_cam, incl, self.fov_y,
                                                      self.width / self.height),
                     self.width, self.height, ThinDisk(r_in, self.r_outer, q),
                     RenderOptions(sky=self.sky, max_steps=self.max_steps,
                                   integrator=self.integrator, row_offset=self.row_offset,
                                   row_step=self.row_step))


class DiffRenderer:
    """A library context running the differentiable render of one DiffScene."""

    def __init__(self, scene: DiffScene | None = None, renderer: Renderer | None = None):
        self.scene = scene or DiffScene()
        self.r = renderer or Renderer(0)
        self._lib = abi.load()

    @property
    def n_values(self) -> int:
        return self.scene.width * self.scene.rows * 3

    def _structs(self, p):
        spin, incl, r_cam, r_in, q = (float(x) for x in p)
        m = Kerr(1.0, spin).to_c()
        d = ThinDisk(r_in, self.scene.r_outer, q).to_c()
        integ = self.scene.integrator.to_c(self.scene.max_steps, abi.GG_PREC_FP64)
        opts = RenderOptions(sky=self.scene.sky, max_steps=self.scene.max_steps,
                             row_offset=self.scene.row_offset,
                             row_step=self.scene.row_step).to_c()
        return m, d, integ, opts, incl, r_cam

    def forward_into(self, p, rgb_dev: int, stream: int = 0) -> None:
        """Forward pass writing width*rows*3 doubles at device address rgb_dev."""
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
        """Forward pass into a new torch tensor (rows, width, 3), float64, CUDA."""
        import torch
        out = torch.empty(self.n_values, dtype=torch.float64, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream
        self.forward_into(p, out.data_ptr(), stream)
        return out.view(self.scene.rows, self.scene.width, 3)


def allreduce_grad(grad, group=None) -> np.ndarray:
    """dL/dp of the whole image from each rank's dL/dp over its rows: the
    sum over the process group (every rank calls it, same order).  A single
    process returns `grad` unchanged."""
    import torch
    import torch.distributed as dist
    g = np.asarray(grad, dtype=np.float64)
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size(group) == 1:
        return g
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.tensor(g, dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy()


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
