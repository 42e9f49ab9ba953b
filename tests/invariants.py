"""First integrals of Kerr geodesics and the capture criterion they give,
restated from the published theory (no code of the reference or of this
repository's kernels): checks of the ray path that do not rest on the
oracle's restatement of the reference.

Boyer-Lindquist coordinates, G = c = 1.  For a geodesic with velocity v:
  E = -(g_tt v^t + g_tphi v^phi),   L = g_tphi v^t + g_phiphi v^phi,
  H = g_mn v^m v^n (the norm, mu^2 = -H),
  Q = (Sigma v^theta)^2 + cos^2 theta (a^2 (mu^2 - E^2) + L^2 / sin^2 theta)
(Carter 1968, Phys. Rev. 174, 1559), all constant along the geodesic.  The
reference's GeodesicRay::from_camera (ray.rs:45-53) sets v^t from the
diagonal terms only, so a Kerr ray's initial H is small but not zero: the
tests use the general-mu form, which holds for any geodesic.

Radial motion: Sigma dr/dlambda = +-sqrt(R(r)) with
  R(r) = (E (r^2 + a^2) - a L)^2 - Delta (mu^2 r^2 + (L - a E)^2 + Q).
A ray that starts at the camera moving inward reaches the horizon iff R > 0
on (r_+, r_cam); otherwise it turns at the largest root and escapes.  The
shadow's rim is where R has a double root: the spherical photon orbits,
whose impact parameters are (Bardeen 1973, in Black Holes, Les Houches;
Chandrasekhar 1983, Mathematical Theory of Black Holes, section 63)
  xi(r)  = -(r^3 - 3 M r^2 + a^2 r + a^2 M) / (a (r - M)),
  eta(r) = -r^3 (r^3 - 6 M r^2 + 9 M^2 r - 4 a^2 M) / (a^2 (r - M)^2),
and for a = 0 the critical impact parameter is b_c = 3 sqrt(3) M.
"""
from __future__ import annotations

import numpy as np


def metric_parts(a: float, M: float, r, th):
    s, c = np.sin(th), np.cos(th)
    s2, c2 = s * s, c * c
    sig = r * r + a * a * c2
    dl = r * r - 2.0 * M * r + a * a
    gtt = -(1.0 - 2.0 * M * r / sig)
    gtp = -2.0 * M * a * r * s2 / sig
    gpp = (r * r + a * a + 2.0 * M * a * a * r * s2 / sig) * s2
    return sig, dl, gtt, gtp, gpp, s2, c2


def invariants(a: float, M: float, x, v):
    """(E, L, Q, H) of states x, v (4 x n each)."""
    sig, dl, gtt, gtp, gpp, s2, c2 = metric_parts(a, M, x[1], x[2])
    vt, vr, vth, vp = v
    E = -(gtt * vt + gtp * vp)
    L = gtp * vt + gpp * vp
    H = gtt * vt * vt + 2.0 * gtp * vt * vp + gpp * vp * vp + (sig / dl) * vr * vr + \
        sig * vth * vth
    Q = (sig * vth) ** 2 + c2 * (a * a * (-H - E * E) + L * L / s2)
    return E, L, Q, H


def drift(a: float, M: float, x0, v0, x1, v1) -> dict:
    """Relative change of each invariant between two states of the same
    rays, each on its natural scale: E on |E|, L on sqrt(L^2 + a^2 E^2), Q on
    L^2 + |Q| + a^2 E^2, H on E^2."""
    E0, L0, Q0, H0 = invariants(a, M, x0, v0)
    E1, L1, Q1, H1 = invariants(a, M, x1, v1)
    ae2 = a * a * E0 * E0
    return {"E": np.abs(E1 - E0) / np.abs(E0),
            "L": np.abs(L1 - L0) / np.sqrt(L0 * L0 + ae2),
            "Q": np.abs(Q1 - Q0) / (L0 * L0 + np.abs(Q0) + ae2),
            "H": np.abs(H1 - H0) / (E0 * E0)}


def radial_coeffs(a: float, M: float, E, L, Q, H):
    """R(r) = c4 r^4 + c3 r^3 + c2 r^2 + c1 r + c0."""
    mu2 = -H
    K = (L - a * E) ** 2 + Q
    w = E * a * a - a * L
    return (E * E - mu2, 2.0 * M * mu2, 2.0 * E * w - (a * a * mu2 + K), 2.0 * M * K,
            w * w - a * a * K)


def capture_margin(a: float, M: float, E, L, Q, H, r_lo: float, r_hi: float):
    """min over r in [r_lo, r_hi] of R(r) / (E^2 r^4): positive for rays the
    hole captures, negative for rays with a radial turning point there, and
    near zero on the shadow's rim (for a = 0 it is 1 - b^2/27 at r = 3M,
    i.e. about 2 (1 - b / b_c) near the rim).  In u = 1/r,
    R / r^4 = c4 + c3 u + c2 u^2 + c1 u^3 + c0 u^4, minimised over its
    stationary points and the interval's ends."""
    c4, c3, c2, c1, c0 = (np.broadcast_to(np.asarray(c, float), np.shape(E))
                          for c in radial_coeffs(a, M, E, L, Q, H))
    E = np.asarray(E, float)
    u_lo, u_hi = 1.0 / r_hi, 1.0 / r_lo
    n = E.size
    # stationary points: 4 c0 u^3 + 3 c1 u^2 + 2 c2 u + c3 = 0
    roots = np.full((n, 3), np.nan + 0j)
    cubic = np.abs(4.0 * c0) > 1e-12 * (np.abs(c1) + np.abs(c2) + np.abs(c3) + 1e-300)
    if cubic.any():
        A = np.zeros((int(cubic.sum()), 3, 3))
        lead = 4.0 * c0[cubic]
        A[:, 0, 0] = -3.0 * c1[cubic] / lead
        A[:, 0, 1] = -2.0 * c2[cubic] / lead
        A[:, 0, 2] = -c3[cubic] / lead
        A[:, 1, 0] = 1.0
        A[:, 2, 1] = 1.0
        roots[cubic] = np.linalg.eigvals(A)
    q = ~cubic  # 3 c1 u^2 + 2 c2 u + c3 = 0
    if q.any():
        qa, qb, qc = 3.0 * c1[q], 2.0 * c2[q], c3[q]
        disc = np.sqrt((qb * qb - 4.0 * qa * qc).astype(complex))
        with np.errstate(divide="ignore", invalid="ignore"):
            roots[q, 0] = np.where(qa != 0.0, (-qb + disc) / (2.0 * qa), -qc / qb)
            roots[q, 1] = np.where(qa != 0.0, (-qb - disc) / (2.0 * qa), np.nan)
    cands = [np.full(n, u_lo), np.full(n, u_hi)]
    for j in range(3):
        uu = roots[:, j]
        ok = np.isfinite(uu) & (np.abs(uu.imag) < 1e-9) & (uu.real > u_lo) & (uu.real < u_hi)
        cands.append(np.where(ok, uu.real, u_hi))
    best = np.full(n, np.inf)
    for uu in cands:
        f = (((c0 * uu + c1) * uu + c2) * uu + c3) * uu + c4
        best = np.minimum(best, f / (E * E))
    return best


def bardeen_critical(a: float, M: float, r):
    """(xi, eta) of the spherical photon orbit at radius r (Bardeen 1973)."""
    xi = -(r ** 3 - 3.0 * M * r * r + a * a * r + a * a * M) / (a * (r - M))
    eta = -r ** 3 * (r ** 3 - 6.0 * M * r * r + 9.0 * M * M * r - 4.0 * a * a * M) / \
        (a * a * (r - M) ** 2)
    return xi, eta


def photon_orbit_radii(a: float, M: float = 1.0) -> tuple[float, float]:
    """Prograde and retrograde circular photon orbits (Bardeen, Press &
    Teukolsky 1972): 2M (1 + cos(2/3 arccos(-+a/M)))."""
    pro = 2.0 * M * (1.0 + np.cos(2.0 / 3.0 * np.arccos(-a / M)))
    retro = 2.0 * M * (1.0 + np.cos(2.0 / 3.0 * np.arccos(a / M)))
    return float(pro), float(retro)
