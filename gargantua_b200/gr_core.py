"""Host mirror of gargantua's ``gr-core`` types on this path.

Names, fields, defaults and error behaviour follow the reference:
``Schwarzschild`` (crates/gr-core/src/schwarzschild.rs:7-23), ``Kerr``
(crates/gr-core/src/kerr.rs:17-34, 53-58) and ``RK45Integrator``
(crates/gr-core/src/geodesic.rs:155-181).  They only carry parameters; all
arithmetic runs in the CUDA library.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

from . import abi


class Schwarzschild:
    """Schwarzschild hole of mass M; ``rs = 2M`` (schwarzschild.rs:12-18)."""

    def __init__(self, mass: float):
        self.mass = float(mass)
        self.rs = 2.0 * self.mass

    @classmethod
    def new(cls, mass: float) -> "Schwarzschild":
        return cls(mass)

    def event_horizon(self) -> float:
        return self.rs

    def to_c(self) -> abi.gg_metric_t:
        m = abi.gg_metric_t()
        m.kind = abi.GG_METRIC_SCHWARZSCHILD
        m.mass = self.mass
        m.spin = 0.0
        return m


class Kerr:
    """Kerr hole in Boyer-Lindquist coordinates (kerr.rs:24-34).

    ``mass <= 0`` raises where the reference asserts; ``|spin| > 0.9999 mass``
    is clamped to ``+-0.9999 mass``.
    """

    def __init__(self, mass: float = 1.0, spin: float = 0.9):
        mass = float(mass)
        if not mass > 0.0:
            raise ValueError("Kerr: mass must be positive")
        max_spin = mass * 0.9999
        spin = float(spin)
        self.mass = mass
        self.spin = min(max(spin, -max_spin), max_spin) if spin == spin else spin

    @classmethod
    def new(cls, mass: float, spin: float) -> "Kerr":
        return cls(mass, spin)

    @classmethod
    def default(cls) -> "Kerr":
        return cls(1.0, 0.9)

    def event_horizon(self) -> float | None:
        d = self.mass * self.mass - self.spin * self.spin
        return None if d < 0.0 else self.mass + d ** 0.5

    def isco(self) -> float:
        """Prograde ISCO radius (Bardeen, Press & Teukolsky 1972)."""
        return abi.load().gg_kerr_isco(self.mass, self.spin)

    def photon_orbit(self) -> float:
        """Prograde circular photon orbit radius."""
        return abi.load().gg_kerr_photon_orbit(self.mass, self.spin)

    def to_c(self) -> abi.gg_metric_t:
        m = abi.gg_metric_t()
        m.kind = abi.GG_METRIC_KERR
        m.mass = self.mass
        m.spin = self.spin
        return m


@dataclass
class RK45Integrator:
    """Adaptive Dormand-Prince stepper parameters (geodesic.rs:155-181).

    ``rtol``/``atol`` extend the reference: with ``rtol > 0`` the velocity
    error is measured as an RMS norm scaled by ``atol + rtol * max(|v|, |v'|)``
    against 1 instead of the absolute ``tolerance``.
    """

    initial_step: float = 0.1
    min_step: float = 1e-8
    max_step: float = 1.0
    tolerance: float = 1e-6
    max_radius: float = 100.0
    horizon_buffer: float = 0.01
    rtol: float = 0.0
    atol: float = 0.0
    # extension: abi.GG_STEPPER_DP45 runs the full Dormand-Prince method on
    # (x, v) instead of the reference's step (see include/gargantua_gpu.h)
    stepper: int = abi.GG_STEPPER_REFERENCE

    def to_c(self, max_steps: int, precision: int = abi.GG_PREC_FP64) -> abi.gg_integrator_t:
        k = abi.gg_integrator_t()
        k.initial_step = self.initial_step
        k.min_step = self.min_step
        k.max_step = self.max_step
        k.tolerance = self.tolerance
        k.max_radius = self.max_radius
        k.horizon_buffer = self.horizon_buffer
        k.rtol = self.rtol
        k.atol = self.atol
        k.max_steps = int(max_steps)
        k.precision = int(precision)
        k.stepper = int(self.stepper)
        return k


def renderer_integrator() -> RK45Integrator:
    """The integrator ``render_inner`` builds (renderer.rs:264): default with r_max = 200."""
    return RK45Integrator(max_radius=200.0)


__all__ = ["Schwarzschild", "Kerr", "RK45Integrator", "renderer_integrator", "C"]
