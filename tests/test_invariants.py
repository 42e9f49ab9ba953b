"""Checks of the ray path against published physics rather than against a
restatement of the reference: conservation of Kerr's first integrals (E,
L_z, Carter's Q and the norm) along traced rays, and the shadow's rim, from
the radial potential's double root (Bardeen 1973) and, for Schwarzschild,
the critical impact parameter 3 sqrt(3) M.  The formulas are in
tests/invariants.py.

The Dormand-Prince forms (the oracle's step_dp45, the FP64 DP45 kernel, the
mixed form) are held to these.  The reference's own step moves the position
by h v_before (geodesic.rs:248, 312), a first-order update: on the 1080p
frame its invariants drift by 1e-3 .. 0.2 and its shadow covers about 7 %
more pixels than the critical curve encloses.  The drop-in reproduces that
algorithm (the parity tests hold it to the oracle), so these checks are not
applied to it."""
from __future__ import annotations

import math

import numpy as np
import pytest

import invariants as inv
from gargantua_b200 import abi, workloads
from gargantua_b200.curved import Camera, CheckerSky, RenderOptions, Scene
from gargantua_b200.gr_core import Kerr, RK45Integrator, Schwarzschild

# drift bounds of the Dormand-Prince forms at rtol 1e-8 (FP64), measured on
# 100,000 seeded rays of the 1080p frame through the oracle: p50 <= 1e-10,
# p99.9 <= 8e-8, max 1e-6
FP64_DRIFT = {"p50": 1e-9, "p99.9": 2e-7, "max": 1e-5}
# the mixed form's FP32 stages leave a drift near FP32's unit roundoff
# (6e-8) times the steps' error growth; its FP64 error estimate and band keep
# the tail where the FP64 form's is
MIXED_DRIFT = {"p50": 2e-7, "p99.9": 2e-6, "max": 1e-5}


def shadow_scene(metric, precision=abi.GG_PREC_FP64, side=96, fov_deg=16.0):
    """The hole seen from r = 50 M at 75 degrees with a 16 degree field of
    view (the shadow fills most of the frame), no disk, the full
    Dormand-Prince stepper at rtol 1e-8 / atol 1e-10."""
    cam = Camera.inclined(50.0, math.radians(75.0), math.radians(fov_deg), 1.0)
    integ = RK45Integrator(max_radius=200.0, rtol=1e-8, atol=1e-10,
                           stepper=abi.GG_STEPPER_DP45)
    return Scene(metric, cam, side, side, None,
                 RenderOptions(sky=CheckerSky(18, 36, 0), max_steps=20000, integrator=integ,
                               precision=precision))


def analytic_classes(scene, oracle_mod):
    """Captured (horizon) or not for every pixel from its initial state's
    invariants, and each pixel's capture margin."""
    a = scene.metric.spin if isinstance(scene.metric, Kerr) else 0.0
    M = scene.metric.mass
    x0, v0 = oracle_mod.initial_states(scene)
    E, L, Q, H = inv.invariants(a, M, x0, v0)
    r_plus = M + math.sqrt(M * M - a * a)
    f = inv.capture_margin(a, M, E, L, Q, H, r_plus, scene.camera.position[1])
    return np.where(f > 0.0, abi.GG_CLASS_HORIZON, abi.GG_CLASS_ESCAPED), f


def check_drift(d: dict, bounds: dict) -> None:
    for name, e in d.items():
        assert np.median(e) <= bounds["p50"], (name, np.median(e))
        assert np.quantile(e, 0.999) <= bounds["p99.9"], (name, np.quantile(e, 0.999))
        assert e.max() <= bounds["max"], (name, e.max())


# ---- the formulas themselves ------------------------------------------------
@pytest.mark.parametrize("a", [0.3, 0.9, 0.998])
def test_bardeen_critical_orbits_are_double_roots(a):
    # every spherical photon orbit between the prograde and retrograde
    # circular ones is a double root of R with E = 1, mu = 0
    pro, retro = inv.photon_orbit_radii(a)
    for r in np.linspace(pro + 1e-3, retro - 1e-3, 25):
        xi, eta = inv.bardeen_critical(a, 1.0, r)
        if eta < 0.0:
            continue
        c4, c3, c2, c1, c0 = inv.radial_coeffs(a, 1.0, 1.0, xi, eta, 0.0)
        R = (((c4 * r + c3) * r + c2) * r + c1) * r + c0
        dR = ((4 * c4 * r + 3 * c3) * r + 2 * c2) * r + c1
        assert abs(R) < 1e-9 * r ** 4 and abs(dR) < 1e-9 * r ** 3, (a, r, R, dR)
        f = inv.capture_margin(a, 1.0, np.array([1.0]), np.array([xi]), np.array([eta]),
                               np.array([0.0]), 1.0 + math.sqrt(1 - a * a) + 1e-9, 50.0)
        assert abs(f[0]) < 1e-9


def test_schwarzschild_critical_impact_parameter():
    # with a = 0 the margin is 1 - b^2/27, zero at b = 3 sqrt(3) M
    b = np.array([5.0, 3.0 * math.sqrt(3.0), 5.3])
    f = inv.capture_margin(0.0, 1.0, np.ones(3), b, np.zeros(3), np.zeros(3), 2.0, 50.0)
    assert np.allclose(f, 1.0 - b * b / 27.0, atol=1e-12)
    assert f[0] > 0.0 > f[2] and abs(f[1]) < 1e-12


# ---- the oracle (CPU) ---------------------------------------------------------
def test_oracle_dp45_conserves_invariants(oracle_mod):
    sc = workloads.kerr_thin_1080p(stepper=abi.GG_STEPPER_DP45)
    idx = np.sort(np.random.default_rng(3).choice(sc.n_samples, 3000, replace=False))
    cr = oracle_mod.trace_cross(sc, idx.astype(np.uint64))
    ok = np.isfinite(cr[0])
    assert ok.mean() > 0.95
    x0, v0 = oracle_mod.initial_states(sc, idx)
    d = inv.drift(sc.metric.spin, 1.0, x0[:, ok], v0[:, ok], cr[:4, ok], cr[4:, ok])
    check_drift(d, FP64_DRIFT)


@pytest.mark.parametrize("metric", [Schwarzschild(1.0), Kerr(1.0, 0.9), Kerr(1.0, 0.998)],
                         ids=["schwarzschild", "kerr0.9", "kerr0.998"])
def test_oracle_dp45_shadow_matches_critical_curve(oracle_mod, metric):
    sc = shadow_scene(metric, side=48)
    want, f = analytic_classes(sc, oracle_mod)
    _, o = oracle_mod.render(sc)
    assert (want == abi.GG_CLASS_HORIZON).mean() > 0.2
    keep = np.abs(f) > 1e-6
    assert keep.mean() > 0.99
    assert np.array_equal(o.cls[keep], want[keep])


# ---- the CUDA kernels -----------------------------------------------------------
@pytest.mark.gpu
def test_fp64_dp45_kernel_conserves_invariants(renderer, oracle_mod):
    # every ray of the 1080p frame that reaches the disk plane or the escape
    # sphere, at its crossing state
    sc = workloads.kerr_thin_1080p(stepper=abi.GG_STEPPER_DP45)
    _, g = renderer.render(sc, rays=True)
    ok = np.isfinite(g.cross[0])
    assert ok.mean() > 0.95
    x0, v0 = oracle_mod.initial_states(sc)
    d = inv.drift(sc.metric.spin, 1.0, x0[:, ok], v0[:, ok], g.cross[:4, ok], g.cross[4:, ok])
    check_drift(d, FP64_DRIFT)


@pytest.mark.gpu
def test_mixed_kernel_conserves_invariants(renderer, oracle_mod):
    # the mixed form on the same frame and crossing states
    sc = workloads.kerr_thin_1080p(precision=abi.GG_PREC_MIXED, stepper=abi.GG_STEPPER_DP45)
    _, g = renderer.render(sc, rays=True)
    ok = np.isfinite(g.cross[0])
    assert ok.mean() > 0.95
    x0, v0 = oracle_mod.initial_states(sc)
    d = inv.drift(sc.metric.spin, 1.0, x0[:, ok], v0[:, ok], g.cross[:4, ok], g.cross[4:, ok])
    check_drift(d, MIXED_DRIFT)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [abi.GG_PREC_FP64, abi.GG_PREC_MIXED], ids=["fp64", "mixed"])
@pytest.mark.parametrize("metric", [Schwarzschild(1.0), Kerr(1.0, 0.9), Kerr(1.0, 0.998)],
                         ids=["schwarzschild", "kerr0.9", "kerr0.998"])
def test_kernel_shadow_matches_critical_curve(renderer, oracle_mod, metric, precision):
    sc = shadow_scene(metric, precision, side=256)
    want, f = analytic_classes(sc, oracle_mod)
    _, g = renderer.render(sc, rays=True)
    keep = np.abs(f) > 1e-6
    assert keep.mean() > 0.99
    bad = np.nonzero(g.cls[keep] != want[keep])[0]
    assert bad.size == 0, f"{bad.size} pixels off the analytic class, margins {f[keep][bad[:5]]}"
