"""Light bending checked against the orbit equation rather than against a
restatement of the reference: the azimuth an equatorial ray sweeps between
the camera and the escape sphere, against the same sweep from the exact
first integrals by quadrature.

For a ray in the equatorial plane of Kerr (Schwarzschild at a = 0) with
energy E, angular momentum L and H = g(v, v) from its initial state (Carter's
Q is 0 there), Boyer-Lindquist's
    dphi/dr = (a (E (r^2 + a^2) - a L) / Delta + L - a E) / sqrt(R(r)),
R the radial potential of tests/invariants.py (Carter 1968).  Between the
camera radius r_c and the escape radius r_e, through the turning point r_0
(the largest root of R), the sweep is the sum of the two legs' integrals
from r_0.  With r = r_0 + s^2 and R = (r - r_0) R_3(r) the integrand is
smooth, so adaptive quadrature gives it to 1e-12.  The traced sweep is phi
at the escape crossing (the camera sits at phi = 0), taken modulo 2 pi: rays
near the critical impact parameter wind round the hole.

The integration error of a ray grows with its sweep's sensitivity to the
impact parameter b, which diverges at the shadow's rim, so each error is
divided by max(1, |b d(sweep)/db|) (central differences of the quadrature)
before it meets the bar.  Rays with L < 0 keep phi near 2 pi, where the
controller's relative tolerance on phi is looser, and show errors about ten
times those of their mirror images.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

import invariants as inv
from gargantua_b200 import abi
from gargantua_b200.curved import Camera, CheckerSky, RenderOptions, Scene
from gargantua_b200.gr_core import Kerr, RK45Integrator, Schwarzschild

R_CAM, R_ESC, WIDTH = 1000.0, 1500.0, 41


def equatorial_scene(metric, precision=abi.GG_PREC_FP64, rtol=1e-10):
    """One row of WIDTH rays in the equatorial plane from r = 1000 M, impact
    parameters up to about 60 M either side, escaping at 1500 M."""
    half = 0.06  # horizontal half-angle, rad
    fov_y = 2.0 * math.atan(math.tan(half) / WIDTH)
    cam = Camera.inclined(R_CAM, math.pi / 2, fov_y, float(WIDTH))
    integ = RK45Integrator(max_radius=R_ESC, max_step=20.0, rtol=rtol, atol=rtol * 1e-2,
                           stepper=abi.GG_STEPPER_DP45)
    return Scene(metric, cam, WIDTH, 1, None,
                 RenderOptions(sky=CheckerSky(18, 36, 0), max_steps=20000, integrator=integ,
                               precision=precision))


def azimuth_sweep(a: float, M: float, E: float, L: float, H: float, r_c: float,
                  r_e: float) -> float:
    from scipy.integrate import quad
    c = np.array(inv.radial_coeffs(a, M, E, L, 0.0, H), float)
    roots = np.roots(c)
    real = roots[np.abs(roots.imag) < 1e-9 * np.abs(roots).max()].real
    r0 = real.max()
    for _ in range(3):  # Newton on the quartic
        r0 -= np.polyval(c, r0) / np.polyval(np.polyder(c), r0)
    cubic = np.polydiv(c, np.array([1.0, -r0]))[0]

    def dphi_ds(s: float) -> float:
        r = r0 + s * s
        d = r * r - 2.0 * M * r + a * a
        phi = a * (E * (r * r + a * a) - a * L) / d + (L - a * E)
        return 2.0 * phi / math.sqrt(np.polyval(cubic, r))

    legs = [quad(dphi_ds, 0.0, math.sqrt(r - r0), epsabs=1e-13, epsrel=1e-13, limit=200)[0]
            for r in (r_c, r_e)]
    return legs[0] + legs[1]


def sweep_errors(scene, x0, v0, cross, cls) -> np.ndarray:
    """Each escaped ray's |traced - exact| sweep over max(1, |b d(sweep)/db|)."""
    a = scene.metric.spin if isinstance(scene.metric, Kerr) else 0.0
    M = scene.metric.mass
    E, L, Q, H = inv.invariants(a, M, x0, v0)
    errs = []
    for k in np.nonzero(cls == abi.GG_CLASS_ESCAPED)[0]:
        assert abs(Q[k]) < 1e-12 * L[k] ** 2 and abs(x0[2, k] - math.pi / 2) < 1e-12
        assert abs(cross[1, k] - R_ESC) < 1e-9 * R_ESC

        def sweep(l):
            return azimuth_sweep(a, M, E[k], l, H[k], R_CAM, R_ESC)
        want = sweep(L[k])
        dl = 1e-6 * abs(L[k])
        sens = abs(L[k] * (sweep(L[k] + dl) - sweep(L[k] - dl)) / (2.0 * dl))
        phi = cross[3, k]
        got = phi + 2.0 * math.pi * round((want - phi) / (2.0 * math.pi))
        errs.append(abs(got - want) / max(1.0, sens))
    return np.array(errs)


METRICS = [Schwarzschild(1.0), Kerr(1.0, 0.5), Kerr(1.0, 0.95)]
IDS = ["schwarzschild", "kerr0.5", "kerr0.95"]


@pytest.mark.parametrize("metric", METRICS, ids=IDS)
def test_oracle_azimuth_sweep_matches_quadrature(oracle_mod, metric):
    sc = equatorial_scene(metric)
    idx = np.arange(WIDTH, dtype=np.uint64)
    x0, v0 = oracle_mod.initial_states(sc)
    cr = oracle_mod.trace_cross(sc, idx)
    _, o = oracle_mod.render(sc)
    escaped = o.cls == abi.GG_CLASS_ESCAPED
    assert escaped.sum() >= WIDTH - 6  # the middle rays fall into the hole
    err = sweep_errors(sc, x0, v0, cr, o.cls)
    assert err.max() < 3e-8, err.max()  # measured 1.2e-8 at rtol 1e-10


@pytest.mark.gpu
@pytest.mark.parametrize("metric", METRICS, ids=IDS)
@pytest.mark.parametrize("precision,rtol,bar", [(abi.GG_PREC_FP64, 1e-10, 3e-8),
                                                (abi.GG_PREC_MIXED, 1e-8, 3e-6)],
                         ids=["fp64", "mixed"])
def test_kernel_azimuth_sweep_matches_quadrature(renderer, oracle_mod, metric, precision, rtol,
                                                 bar):
    sc = equatorial_scene(metric, precision, rtol)
    x0, v0 = oracle_mod.initial_states(sc)
    _, g = renderer.render(sc, rays=True)
    assert (g.cls == abi.GG_CLASS_ESCAPED).sum() >= WIDTH - 6
    err = sweep_errors(sc, x0, v0, g.cross, g.cls)
    assert err.max() < bar, err.max()
