"""The reference's own known-answer tests, run on the CPU oracle.

Each test restates one test of gargantua with its points and tolerances:
crates/gr-core/src/{geodesic,schwarzschild,kerr}.rs ``mod tests`` and
crates/gr-renderer/tests/render_sanity.rs.  Passing them pins the oracle to
everything the reference's test suite pins for this path.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import pytest

from gargantua_b200 import abi
from gargantua_b200.curved import Camera, RenderOptions, Scene
from gargantua_b200.gr_core import Kerr, Schwarzschild

PI = math.pi


def ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def metric_tensor(L, metric, pos):
    g = np.zeros(16)
    m = metric.to_c()
    assert L.ggo_metric_tensor(C.byref(m), ptr(np.asarray(pos, float)), ptr(g)) == 0
    return g.reshape(4, 4)


def test_circular_orbit(oracle_mod):
    """geodesic.rs:361-389: RK4 h=0.01, Schwarzschild r=6 circular, one period."""
    L = oracle_mod.lib()
    r = 6.0
    omega = math.sqrt(1.0 / (r * r * r))
    st = np.array([0.0, r, PI / 2.0, 0.0, 1.0, 0.0, 0.0, omega, 0.0])
    steps = int((2.0 * PI / omega) / 0.01)
    m = Schwarzschild(1.0).to_c()
    assert L.ggo_rk4_run(C.byref(m), ptr(st), 0.01, steps) == 0
    assert abs(st[1] - r) < 0.1, st[1]


def test_keplerian_orbit_is_normalized_timelike(oracle_mod):
    """schwarzschild.rs:162-170."""
    L = oracle_mod.lib()
    metric = Schwarzschild(1.0)
    pos = np.array([0.0, 10.0, PI / 2.0, 0.0])
    u = np.zeros(4)
    m = metric.to_c()
    assert L.ggo_orbital_four_velocity(C.byref(m), ptr(pos), ptr(u)) == 1
    g = metric_tensor(L, metric, pos)
    norm = (g @ u) @ u
    assert abs(norm + 1.0) < 1e-9
    assert u[3] > 0.0


def test_no_circular_orbit_inside_photon_sphere(oracle_mod):
    """schwarzschild.rs:173-177."""
    L = oracle_mod.lib()
    m = Schwarzschild(1.0).to_c()
    u = np.zeros(4)
    assert L.ggo_orbital_four_velocity(C.byref(m), ptr(np.array([0.0, 2.5, PI / 2, 0.0])),
                                       ptr(u)) == 0


def test_schwarzschild_flat_at_infinity(oracle_mod):
    """schwarzschild.rs:180-188."""
    g = metric_tensor(oracle_mod.lib(), Schwarzschild(1.0), [0.0, 1000.0, PI / 2, 0.0])
    assert abs(g[0, 0] + 1.0) < 0.01
    assert abs(g[1, 1] - 1.0) < 0.01


def test_kerr_reduces_to_schwarzschild_when_a_is_zero(oracle_mod):
    """kerr.rs:508-537, EPS = 1e-12."""
    L = oracle_mod.lib()
    for pos in ([0.0, 10.0, PI / 3, 0.0], [0.0, 6.0, PI / 2, 1.0], [1.0, 20.0, PI / 4, 2.5],
                [0.0, 5.0, 2.0, 0.5]):
        gk = metric_tensor(L, Kerr(1.0, 0.0), pos)
        gs = metric_tensor(L, Schwarzschild(1.0), pos)
        assert np.all(np.abs(gk - gs) < 1e-12)


def test_kerr_horizon(oracle_mod):
    """kerr.rs:541-550."""
    rh = C.c_double()
    m = Kerr(1.0, 0.5).to_c()
    assert oracle_mod.lib().ggo_event_horizon(C.byref(m), C.byref(rh)) == 1
    assert abs(rh.value - (1.0 + math.sqrt(0.75))) < 1e-12


def test_kerr_christoffel_matches_numerical(oracle_mod):
    """kerr.rs:554-575: analytic vs central-difference (h=1e-5) to 1e-4."""
    L = oracle_mod.lib()
    m = Kerr(1.0, 0.7).to_c()
    pos = np.array([0.0, 10.0, PI / 3, 0.7])
    an = np.zeros(64)
    nu = np.zeros(64)
    assert L.ggo_christoffel(C.byref(m), ptr(pos), ptr(an)) == 0
    assert L.ggo_numerical_christoffel(C.byref(m), ptr(pos), 1e-5, ptr(nu)) == 0
    assert np.all(np.abs(an - nu) < 1e-4), np.abs(an - nu).max()


def test_kerr_circular_orbit_equatorial(oracle_mod):
    """kerr.rs:579-610: RK4 h=0.05, a=0.5, r=10, drift < 0.5."""
    L = oracle_mod.lib()
    k = Kerr(1.0, 0.5)
    r0 = 10.0
    omega = math.sqrt(k.mass) / (r0 ** 1.5 + k.spin * math.sqrt(k.mass))
    st = np.array([0.0, r0, PI / 2, 0.0, 1.0, 0.0, 0.0, omega, 0.0])
    steps = int((2 * PI / omega) / 0.05)
    m = k.to_c()
    assert L.ggo_rk4_run(C.byref(m), ptr(st), 0.05, steps) == 0
    assert abs(st[1] - r0) < 0.5


def test_kerr_metric_signature_and_symmetry(oracle_mod):
    """kerr.rs:614-629."""
    g = metric_tensor(oracle_mod.lib(), Kerr(1.0, 0.9), [0.0, 10.0, PI / 2, 0.0])
    assert g[0, 0] < 0 and g[1, 1] > 0 and g[2, 2] > 0 and g[3, 3] > 0
    assert abs(g[0, 3] - g[3, 0]) < 1e-12
    assert abs(g[0, 3]) > 1e-10


def test_horizon_shadow_and_escape(oracle_mod):
    """gr-renderer/tests/render_sanity.rs:16-27: 32x24 has black and non-black pixels."""
    scene = Scene(Schwarzschild(1.0), Camera(aspect=32 / 24), 32, 24, None, RenderOptions())
    img, _ = oracle_mod.render(scene)
    px = img.reshape(-1, 3)
    assert (px == 0).all(axis=1).any()
    assert (px != 0).any(axis=1).any()


def test_kerr_spin_clamp_and_mass_assert():
    """kerr.rs:29-34: |a| clamped to 0.9999 M; mass <= 0 is rejected."""
    assert Kerr(1.0, 1.5).spin == pytest.approx(0.9999)
    assert Kerr(2.0, -5.0).spin == pytest.approx(-1.9998)
    with pytest.raises(ValueError):
        Kerr(0.0, 0.5)


def test_procedural_sky_hash(oracle_mod):
    """sky.rs:26-40 restated with Python integers for a few directions."""
    import struct
    L = oracle_mod.lib()
    mask = (1 << 64) - 1

    def expect(d):
        def h(x):
            b = struct.unpack("<Q", struct.pack("<d", x))[0]
            return (b * 6364136223846793005 + 1442695040888963407) & mask

        def rotl(x, k):
            return ((x << k) | (x >> (64 - k))) & mask
        hv = h(d[0]) ^ rotl(h(d[1]), 17) ^ rotl(h(d[2]), 34)
        if hv % 512 < 3:
            b = (180 + hv % 75) / 255.0
            return [b, b, b]
        return [0.0, 0.0, 10.0 / 255.0 + abs(d[2]) * 15.0 / 255.0]

    rng = np.random.default_rng(7)
    stars = 0
    for _ in range(4000):
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        out = np.zeros(3)
        L.ggo_procedural_sky(ptr(d), ptr(out))
        e = expect(list(d))
        assert list(out) == e
        stars += out[0] > 0
    assert 5 < stars < 60  # about 3/512 of directions are stars


def test_encode_srgb(oracle_mod):
    """renderer.rs:69-80 at the piecewise boundary, clamps and rounding."""
    L = oracle_mod.lib()
    cases = {0.0: 0, 1.0: 255, 2.0: 255, -1.0: 0, 0.0031308: round(12.92 * 0.0031308 * 255),
             0.5: round((1.055 * 0.5 ** (1 / 2.4) - 0.055) * 255)}
    for lin, want in cases.items():
        out = np.zeros(3, np.uint8)
        L.ggo_encode_srgb(ptr(np.array([lin, lin, lin])), ptr(out))
        assert out[0] == want, (lin, out[0], want)


def test_rearranged_kerr_rhs_matches_dense(oracle_mod):
    """The Kerr right-hand side folded into the contraction (one reciprocal,
    shared row factors) equals the reference's dense Christoffel contraction
    (metric.rs:37-52) to rounding, at random points and spins."""
    dense, alt = oracle_mod.lib(), oracle_mod.lib("alt")
    rng = np.random.default_rng(3)
    worst = 0.0
    for _ in range(500):
        k = Kerr(1.0, rng.uniform(-0.998, 0.998))
        r = rng.uniform(k.event_horizon() + 0.05, 200.0)
        pos = np.array([0.0, r, rng.uniform(0.05, PI - 0.05), 0.3])
        vel = rng.normal(size=4)
        a1, a2 = np.zeros(4), np.zeros(4)
        m = k.to_c()
        dense.ggo_geodesic_acceleration(C.byref(m), ptr(pos), ptr(vel), ptr(a1))
        alt.ggo_geodesic_acceleration(C.byref(m), ptr(pos), ptr(vel), ptr(a2))
        worst = max(worst, np.abs(a1 - a2).max() / np.abs(a1).max())
    assert worst < 1e-12, worst
