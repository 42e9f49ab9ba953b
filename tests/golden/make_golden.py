"""Generates tests/golden/golden_rays.json from a pure-Python restatement.

This is a second, independent restatement of gargantua's f64 ray path, written
straight from the Rust source in plain Python floats (IEEE double, no fused
multiply-add, ``math`` = the platform libm like Rust's ``f64`` methods).  The
C++ oracle (oracle/gg_oracle.hpp) must reproduce these vectors, which pins it
against restatement slips; the reference itself cannot run here (Rust, no
toolchain).

    python tests/golden/make_golden.py       # rewrites golden_rays.json

Reference files: crates/gr-core/src/{metric,schwarzschild,kerr,geodesic}.rs and
crates/raytracer/src/curved/{camera,ray,tracer,disk,sky,renderer}.rs.
"""
from __future__ import annotations

import json
import math
import struct
from pathlib import Path

PI = math.pi
OUT = Path(__file__).resolve().parent / "golden_rays.json"


# ---- metrics ---------------------------------------------------------------
class Schw:
    def __init__(self, mass):
        self.mass, self.rs = mass, 2.0 * mass

    def g(self, pos):  # schwarzschild.rs:26-43
        r = max(pos[1], 1e-10)
        f = 1.0 - self.rs / r
        s = math.sin(pos[2])
        return {"tt": -f, "rr": 1.0 / f, "thth": r * r, "phph": r * r * s * s, "tph": 0.0}

    def acc(self, pos, vel):  # schwarzschild.rs:99-140
        r = max(pos[1], 1e-10)
        s, c = math.sin(pos[2]), math.cos(pos[2])
        rs = self.rs
        f_denom = r * (r - rs)
        rmrs = r - rs
        inv_r = 1.0 / r
        g_t_tr = rs / (2.0 * f_denom)
        g_r_tt = rs * rmrs / (2.0 * r * r * r)
        g_r_rr = -rs / (2.0 * f_denom)
        g_r_thth = -rmrs
        g_r_phph = -rmrs * s * s
        g_th_phph = -s * c
        g_ph_thph = c / s
        vt, vr, vth, vph = vel
        return [-2.0 * g_t_tr * vt * vr,
                -g_r_tt * vt * vt - g_r_rr * vr * vr - g_r_thth * vth * vth
                - g_r_phph * vph * vph,
                -2.0 * inv_r * vr * vth - g_th_phph * vph * vph,
                -2.0 * inv_r * vr * vph - 2.0 * g_ph_thph * vth * vph]

    def horizon(self):
        return self.rs

    def orbit(self, pos):  # schwarzschild.rs:146-153
        r = pos[1]
        if r <= 3.0 * self.mass:
            return None
        return circular(self, pos, math.sqrt(self.mass / (r * r * r)))


class Kerr:
    def __init__(self, mass, spin):  # kerr.rs:29-34
        ms = mass * 0.9999
        self.mass, self.spin = mass, min(max(spin, -ms), ms)

    def sigma(self, r, th):
        a = self.spin
        c = math.cos(th)
        return r * r + a * a * c * c

    def delta(self, r):
        m, a = self.mass, self.spin
        return r * r - 2.0 * m * r + a * a

    def g(self, pos):  # kerr.rs:61-94
        r = max(pos[1], 1e-10)
        th = pos[2]
        m, a = self.mass, self.spin
        a2 = a * a
        sig, dl = self.sigma(r, th), self.delta(r)
        s = math.sin(th)
        s2 = s * s
        return {"tt": -(1.0 - 2.0 * m * r / sig), "rr": sig / dl, "thth": sig,
                "phph": (r * r + a2 + 2.0 * m * a2 * r * s2 / sig) * s2,
                "tph": -2.0 * m * a * r * s2 / sig}

    def christoffel(self, pos):  # kerr.rs:100-424
        r = max(pos[1], 1e-10)
        th = pos[2]
        m, a = self.mass, self.spin
        a2 = a * a
        sig, dl = self.sigma(r, th), self.delta(r)
        s, c = math.sin(th), math.cos(th)
        s2 = s * s
        sig2 = sig * sig
        r2 = r * r
        ds_r = 2.0 * r
        ds_th = -2.0 * a2 * s * c
        dd_r = 2.0 * r - 2.0 * m
        rpa = r2 + a2
        big_a = rpa * rpa - a2 * dl * s2
        gi_tt = -big_a / (sig * dl)
        gi_tp = -2.0 * m * a * r / (sig * dl)
        gi_rr = dl / sig
        gi_hh = 1.0 / sig
        gi_pp = (dl - a2 * s2) / (sig * dl * s2)
        dtt_r = 2.0 * m / sig - 2.0 * m * r * ds_r / sig2
        dtt_h = -2.0 * m * r * ds_th / sig2
        drr_r = (ds_r * dl - sig * dd_r) / (dl * dl)
        drr_h = ds_th / dl
        dhh_r = ds_r
        dhh_h = ds_th
        big_p = 2.0 * m * a2 * r
        dpp_r = 2.0 * r * s2 + s2 * s2 * 2.0 * m * a2 * (sig - 2.0 * r2) / sig2
        dpp_h = 2.0 * rpa * s * c + big_p * (4.0 * s * s * s * c * sig - s2 * s2 * ds_th) / sig2
        dtp_r = -2.0 * m * a * s2 * (sig - r * ds_r) / sig2
        dtp_h = -2.0 * m * a * r * (2.0 * s * c * sig - s2 * ds_th) / sig2
        G = [[[0.0] * 4 for _ in range(4)] for _ in range(4)]

        def sym(mu, i, j, v):
            G[mu][i][j] = v
            G[mu][j][i] = v
        sym(0, 0, 1, 0.5 * (gi_tt * dtt_r + gi_tp * dtp_r))
        sym(0, 0, 2, 0.5 * (gi_tt * dtt_h + gi_tp * dtp_h))
        sym(0, 1, 3, 0.5 * (gi_tt * dtp_r + gi_tp * dpp_r))
        sym(0, 2, 3, 0.5 * (gi_tt * dtp_h + gi_tp * dpp_h))
        G[1][0][0] = -0.5 * gi_rr * dtt_r
        G[1][1][1] = 0.5 * gi_rr * drr_r
        G[1][2][2] = -0.5 * gi_rr * dhh_r
        G[1][3][3] = -0.5 * gi_rr * dpp_r
        sym(1, 1, 2, 0.5 * gi_rr * drr_h)
        sym(1, 0, 3, -0.5 * gi_rr * dtp_r)
        G[2][0][0] = -0.5 * gi_hh * dtt_h
        G[2][1][1] = -0.5 * gi_hh * drr_h
        G[2][2][2] = 0.5 * gi_hh * dhh_h
        G[2][3][3] = -0.5 * gi_hh * dpp_h
        sym(2, 1, 2, 0.5 * gi_hh * dhh_r)
        sym(2, 0, 3, -0.5 * gi_hh * dtp_h)
        sym(3, 0, 1, 0.5 * (gi_tp * dtt_r + gi_pp * dtp_r))
        sym(3, 0, 2, 0.5 * (gi_tp * dtt_h + gi_pp * dtp_h))
        sym(3, 1, 3, 0.5 * (gi_tp * dtp_r + gi_pp * dpp_r))
        sym(3, 2, 3, 0.5 * (gi_tp * dtp_h + gi_pp * dpp_h))
        return G

    def acc(self, pos, vel):  # metric.rs:37-52
        G = self.christoffel(pos)
        out = [0.0, 0.0, 0.0, 0.0]
        for mu in range(4):
            for al in range(4):
                for be in range(4):
                    out[mu] = out[mu] - G[mu][al][be] * vel[al] * vel[be]
        return out

    def horizon(self):
        d = self.mass * self.mass - self.spin * self.spin
        return None if d < 0.0 else self.mass + math.sqrt(d)

    def orbit(self, pos):  # kerr.rs:439-449
        r = pos[1]
        if r <= 0.0:
            return None
        sm = math.sqrt(self.mass)
        return circular(self, pos, sm / (r ** 1.5 + self.spin * sm))


def circular(metric, pos, omega):  # metric.rs:82-94
    g = metric.g(pos)
    denom = -(g["tt"] + 2.0 * g["tph"] * omega + g["phph"] * omega * omega)
    if denom <= 0.0 or not math.isfinite(denom):
        return None
    ut = 1.0 / math.sqrt(denom)
    return [ut, 0.0, 0.0, omega * ut]


# ---- RK45 (geodesic.rs:185-352) ----------------------------------------------
A2, A3, A4, A5 = 1.0 / 5.0, 3.0 / 10.0, 4.0 / 5.0, 8.0 / 9.0
B21 = 1.0 / 5.0
B31, B32 = 3.0 / 40.0, 9.0 / 40.0
B41, B42, B43 = 44.0 / 45.0, -56.0 / 15.0, 32.0 / 9.0
B51, B52, B53, B54 = 19372.0 / 6561.0, -25360.0 / 2187.0, 64448.0 / 6561.0, -212.0 / 729.0
B61, B62, B63, B64, B65 = (9017.0 / 3168.0, -355.0 / 33.0, 46732.0 / 5247.0, 49.0 / 176.0,
                           -5103.0 / 18656.0)
C1, C3, C4, C5, C6 = 35.0 / 384.0, 500.0 / 1113.0, 125.0 / 192.0, -2187.0 / 6784.0, 11.0 / 84.0
D1, D3, D4, D5, D6, D7 = (5179.0 / 57600.0, 7571.0 / 16695.0, 393.0 / 640.0,
                          -92097.0 / 339200.0, 187.0 / 2100.0, 1.0 / 40.0)


def vadd(a, b):
    return [a[i] + b[i] for i in range(4)]


def vscale(s, v):
    return [s * v[i] for i in range(4)]


def lin(*terms):
    """Left-associated sum of coefficient * vector terms."""
    acc = vscale(terms[0][0], terms[0][1])
    for c, v in terms[1:]:
        acc = vadd(acc, vscale(c, v))
    return acc


def valid(p):
    return all(math.isfinite(x) for x in p) and p[1] > 0.0


def normalize(p):
    p = list(p)
    if p[2] < 0.0:
        p[2] = -p[2]
        p[3] = p[3] + PI
    if p[2] > PI:
        p[2] = 2.0 * PI - p[2]
        p[3] = p[3] + PI
    m = math.fmod(p[3], 2.0 * PI)
    p[3] = m + 2.0 * PI if m < 0.0 else m
    return p


def rk45_step(metric, I, st, h):
    """Returns (result, h_new, accepted, h_used); st is mutated."""
    pos, vel = st["x"], st["v"]
    if pos[1] > I["max_radius"]:
        return "esc", h, False, 0.0
    rh = metric.horizon()
    if rh is not None and (pos[1] < rh + I["horizon_buffer"] or pos[1] < rh):
        return "hor", h, False, 0.0
    k1 = metric.acc(pos, vel)
    p2 = vadd(pos, vscale(h * A2, vel))
    v2 = vadd(vel, vscale(h * B21, k1))
    if not valid(p2):
        return "cont", h * 0.5, False, 0.0
    k2 = metric.acc(p2, v2)
    p3 = vadd(pos, vscale(h * A3, vel))
    v3 = vadd(vel, vscale(h, lin((B31, k1), (B32, k2))))
    if not valid(p3):
        return "cont", h * 0.5, False, 0.0
    k3 = metric.acc(p3, v3)
    p4 = vadd(pos, vscale(h * A4, vel))
    v4 = vadd(vel, vscale(h, lin((B41, k1), (B42, k2), (B43, k3))))
    if not valid(p4):
        return "cont", h * 0.5, False, 0.0
    k4 = metric.acc(p4, v4)
    p5 = vadd(pos, vscale(h * A5, vel))
    v5 = vadd(vel, vscale(h, lin((B51, k1), (B52, k2), (B53, k3), (B54, k4))))
    if not valid(p5):
        return "cont", h * 0.5, False, 0.0
    k5 = metric.acc(p5, v5)
    p6 = vadd(pos, vscale(h, vel))
    v6 = vadd(vel, vscale(h, lin((B61, k1), (B62, k2), (B63, k3), (B64, k4), (B65, k5))))
    if not valid(p6):
        return "cont", h * 0.5, False, 0.0
    k6 = metric.acc(p6, v6)
    nv = vadd(vel, vscale(h, lin((C1, k1), (C3, k3), (C4, k4), (C5, k5), (C6, k6))))
    k7 = metric.acc(p6, nv)
    ve = vadd(vel, vscale(h, lin((D1, k1), (D3, k3), (D4, k4), (D5, k5), (D6, k6), (D7, k7))))
    if I["rtol"] > 0.0:
        s = 0.0
        for i in range(4):
            sc = I["atol"] + I["rtol"] * max(abs(vel[i]), abs(nv[i]))
            q = (nv[i] - ve[i]) / sc
            s = s + q * q
        err, tol = math.sqrt(s * 0.25), 1.0
    else:
        d = [nv[i] - ve[i] for i in range(4)]
        s = d[0] * d[0]
        s = s + d[1] * d[1]
        s = s + d[2] * d[2]
        s = s + d[3] * d[3]
        err, tol = math.sqrt(s), I["tolerance"]
    if err < tol or h <= I["min_step"]:
        st["x"] = normalize(vadd(pos, vscale(h, vel)))
        st["v"] = nv
        st["lam"] = st["lam"] + h
        hn = h
        if err > 0.0:
            hn = min(max(h * 0.9 * (tol / err) ** 0.2, I["min_step"]), I["max_step"])
        return "cont", hn, True, h
    return "cont", max(h * 0.9 * (tol / err) ** 0.25, I["min_step"]), False, 0.0


# ---- camera / rays ---------------------------------------------------------------
def dot3(a, b):
    s = a[0] * b[0]
    s = s + a[1] * b[1]
    return s + a[2] * b[2]


def normalize3(v):
    n = math.sqrt(dot3(v, v))
    return [v[0] / n, v[1] / n, v[2] / n]


def cross3(a, b):
    return [a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]]


def pixel_direction(cam, u, v):  # camera.rs:20-29
    f = normalize3(cam["look_at"])
    r = normalize3(cross3(f, cam["up"]))
    up = normalize3(cross3(r, f))
    hh = math.tan(cam["fov"] / 2.0)
    hw = hh * cam["aspect"]
    d = [(f[i] + (u * hw) * r[i]) + (v * hh) * up[i] for i in range(3)]
    return normalize3(d)


def from_camera(metric, cam, u, v):  # ray.rs:14-61
    n = pixel_direction(cam, u, v)
    pos = list(cam["pos"])
    st, ct = math.sin(pos[2]), math.cos(pos[2])
    sp, cp = math.sin(pos[3]), math.cos(pos[3])
    nr = dot3(n, [st * cp, st * sp, ct])
    nt = dot3(n, [ct * cp, ct * sp, -st])
    npp = dot3(n, [-sp, cp, 0.0])
    g = metric.g(pos)
    kr = nr / math.sqrt(g["rr"])
    kth = nt / math.sqrt(g["thth"])
    kph = npp / math.sqrt(g["phph"])
    sns = g["rr"] * kr * kr + g["thth"] * kth * kth + g["phph"] * kph * kph
    return {"x": pos, "v": [math.sqrt(-sns / g["tt"]), kr, kth, kph], "lam": 0.0}


def redshift(metric, pos, p, sq_obs):  # tracer.rs:158-183
    g = metric.g(pos)
    p_t = g["tt"] * p[0] + g["tph"] * p[3]
    e_obs = max(-p_t / sq_obs, 0.0)
    u = metric.orbit(pos)
    if u is not None:
        p_phi = g["tph"] * p[0] + g["phph"] * p[3]
        e_emit = max(-(p_t * u[0] + p_phi * u[3]), 0.0)
    else:
        gt = -g["tt"]
        e_emit = max(-p_t / math.sqrt(gt) if gt > 0.0 else 0.0, 0.0)
    return e_obs / e_emit if e_emit > 0.0 else 0.0


def density(D, pos):  # disk.rs:40-59
    r, th = pos[1], pos[2]
    s, c = math.sin(th), math.cos(th)
    R = r * abs(s)
    z = r * c
    if R < D["r_inner"] or R > D["r_outer"]:
        return 0.0
    q = D["r_inner"] / R
    return D["density_0"] * (q * q) * math.exp(-z * z / (2.0 * D["scale_height"] * D["scale_height"]))


def emission(D, pos):  # disk.rs:65-81
    rho = density(D, pos)
    if rho == 0.0:
        return 0.0
    R = pos[1] * abs(math.sin(pos[2]))
    if R < D["r_inner"]:
        return 0.0
    return rho * rho * (D["r_inner"] / R) ** 0.75


MASK = (1 << 64) - 1


def splitmix64(x):
    x = (x + 0x9E3779B97F4A7C15) & MASK
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & MASK
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & MASK
    return x ^ (x >> 31)


def procedural_sky(d):  # sky.rs:26-40
    def hsh(x):
        bits = struct.unpack("<Q", struct.pack("<d", x))[0]
        return (bits * 6364136223846793005 + 1442695040888963407) & MASK

    def rotl(x, k):
        return ((x << k) | (x >> (64 - k))) & MASK
    h = hsh(d[0]) ^ rotl(hsh(d[1]), 17) ^ rotl(hsh(d[2]), 34)
    if h % 512 < 3:
        b = float(180 + h % 75) / 255.0
        return [b, b, b]
    return [0.0, 0.0, 10.0 / 255.0 + abs(d[2]) * 15.0 / 255.0]


def checker_sky(theta, phi, rows, cols, seed):
    i = min(max(math.floor(theta / (PI / rows)), 0), rows - 1)
    j = min(max(math.floor(phi / ((2.0 * PI) / cols)), 0), cols - 1)
    z = splitmix64(seed ^ splitmix64(i * cols + j))
    base = 0.9 if (i + j) & 1 else 0.1
    return [base * (0.75 + 0.25 * (float((z >> (21 * k)) & 0x1FFFFF) * (1.0 / 2097152.0)))
            for k in range(3)]


def spatial_dir(v):  # tracer.rs:185-189
    s = [v[1], v[2], v[3]]
    n = math.sqrt(dot3(s, s))
    return [s[0] / n, s[1] / n, s[2] / n] if n > 0.0 else [1.0, 0.0, 0.0]


def disk_color(I):  # renderer.rs:62-66
    x = I / (1.0 + I)
    return [x ** 0.5, x ** 1.2, x ** 2.5]


def trace(metric, S, cam, st):
    I = S["integ"]
    h = I["initial_step"]
    inten, trans = 0.0, 1.0
    gobs = metric.g(cam["pos"])
    sq = math.sqrt(max(-gobs["tt"], 0.0))
    att = acc = 0
    res = {"cls": 3}
    for _ in range(S["max_steps"]):
        xb, vb, lb = list(st["x"]), list(st["v"]), st["lam"]
        result, h, accepted, hu = rk45_step(metric, I, st, h)
        att += 1
        acc += accepted
        if accepted and S["disk"] and S["disk"]["kind"] == "thin":
            D = S["disk"]
            db, da = xb[2] - PI / 2.0, st["x"][2] - PI / 2.0
            if (db < 0.0 and da >= 0.0) or (db > 0.0 and da <= 0.0):
                s = db / (db - da)
                raw_r = xb[1] + hu * vb[1]
                rc = xb[1] + s * (raw_r - xb[1])
                if D["r_inner"] <= rc <= D["r_outer"]:
                    vc = [vb[i] + s * (st["v"][i] - vb[i]) for i in range(4)]
                    g = redshift(metric, [0.0, rc, PI / 2.0, 0.0], vc, sq)
                    q = D["r_inner"] / rc
                    g2 = g * g
                    xc = normalize([xb[i] + s * ((xb[i] + hu * vb[i]) - xb[i]) for i in range(4)])
                    xc[1], xc[2] = rc, PI / 2.0
                    res.update(cls=2, intensity=(g2 * g2) * q ** D["q"], color_temp=g * q ** 0.75,
                               x=xc, v=vc, lam=lb + s * hu)
                    res["rgb"] = disk_color(res["intensity"])
                    break
        if S["disk"] and S["disk"]["kind"] == "vol":
            D = S["disk"]
            dl = max(st["lam"] - lb, 0.0)
            if dl > 0.0:
                mid = [0.5 * (xb[i] + st["x"][i]) for i in range(4)]
                rho = density(D, mid)
                if rho > 0.0:
                    j = emission(D, mid)
                    gf = redshift(metric, mid, [0.5 * (vb[i] + st["v"][i]) for i in range(4)], sq)
                    g2 = gf * gf
                    inten = inten + j * (g2 * g2) * dl * trans
                    trans = trans * math.exp(-rho * dl * 0.1)
                    if trans < 1e-3:
                        res.update(cls=2, intensity=inten)
                        break
            if result != "cont":
                res["cls"] = 2 if inten > 0.0 else (1 if result == "esc" else 0)
                if inten > 0.0:
                    res["intensity"] = inten
                break
        else:
            if result == "hor":
                res["cls"] = 0
                break
            if result == "esc":
                res["cls"] = 1
                break
    else:
        if S["disk"] and S["disk"]["kind"] == "vol" and inten > 0.0:
            res.update(cls=2, intensity=inten)
    res.setdefault("x", st["x"])
    res.setdefault("v", st["v"])
    res.setdefault("lam", st["lam"])
    res["attempts"], res["accepted"] = att, acc
    if "rgb" not in res:
        c = res["cls"]
        if c == 0:
            res["rgb"] = [0.0, 0.0, 0.0]
        elif c == 1:
            if S["sky"] == "checker":
                res["rgb"] = checker_sky(st["x"][2], st["x"][3], 18, 36, S["sky_seed"])
            else:
                res["rgb"] = procedural_sky(spatial_dir(st["v"]))
        elif c == 2:
            res["rgb"] = disk_color(res["intensity"])
        else:
            res["rgb"] = [0.0, 0.0, 10.0 / 255.0]
    res.setdefault("intensity", 0.0)
    return res


# ---- cases -------------------------------------------------------------------------
def cases():
    ref_integ = {"initial_step": 0.1, "min_step": 1e-8, "max_step": 1.0, "tolerance": 1e-6,
                 "max_radius": 200.0, "horizon_buffer": 0.01, "rtol": 0.0, "atol": 0.0}
    cfg_integ = dict(ref_integ, rtol=1e-8, atol=1e-10)
    cli_cam = {"pos": [0.0, 30.0, PI / 2.0, 0.0], "look_at": [-1.0, 0.0, 0.0],
               "up": [0.0, 0.0, 1.0], "fov": 60.0 * (PI / 180.0)}

    def inclined(r, inc_deg, aspect):
        inc = inc_deg * (PI / 180.0)
        return {"pos": [0.0, r, inc, 0.0], "look_at": [-math.sin(inc), 0.0, -math.cos(inc)],
                "up": [0.0, 0.0, 1.0], "fov": 60.0 * (PI / 180.0), "aspect": aspect}

    a09 = 0.9
    z1 = 1 + (1 - a09 * a09) ** (1 / 3) * ((1 + a09) ** (1 / 3) + (1 - a09) ** (1 / 3))
    z2 = math.sqrt(3 * a09 * a09 + z1 * z1)
    isco = 3 + z2 - math.sqrt((3 - z1) * (3 + z1 + 2 * z2))
    yield {"name": "cli_schwarzschild_32x24", "metric": ["schw", 1.0, 0.0],
           "cam": dict(cli_cam, aspect=32 / 24), "w": 32, "h": 24, "integ": ref_integ,
           "max_steps": 5000, "disk": None, "sky": "procedural", "sky_seed": 0,
           "pixels": [[0, 0], [16, 12], [15, 11], [31, 23], [20, 5], [8, 18]]}
    yield {"name": "cli_kerr09_volumetric_64x48", "metric": ["kerr", 1.0, 0.9],
           "cam": dict(cli_cam, aspect=64 / 48), "w": 64, "h": 48, "integ": ref_integ,
           "max_steps": 5000,
           "disk": {"kind": "vol", "r_inner": 6.0, "r_outer": 20.0, "scale_height": 1.0,
                    "density_0": 1.0},
           "sky": "procedural", "sky_seed": 0,
           "pixels": [[32, 24], [10, 24], [50, 26], [32, 10], [5, 5], [40, 30]]}
    yield {"name": "c1_schwarzschild_thin_256", "metric": ["schw", 1.0, 0.0],
           "cam": inclined(30.0, 80.0, 1.0), "w": 256, "h": 256, "integ": cfg_integ,
           "max_steps": 10000,
           "disk": {"kind": "thin", "r_inner": 6.0, "r_outer": 20.0, "q": 3.0},
           "sky": "checker", "sky_seed": 0,
           "pixels": [[128, 128], [100, 128], [60, 140], [200, 90], [10, 10], [128, 170]]}
    yield {"name": "c2_kerr09_thin_1080p", "metric": ["kerr", 1.0, 0.9],
           "cam": inclined(50.0, 75.0, 1920 / 1080), "w": 1920, "h": 1080, "integ": cfg_integ,
           "max_steps": 10000,
           "disk": {"kind": "thin", "r_inner": isco, "r_outer": 30.0, "q": 3.0},
           "sky": "checker", "sky_seed": 0,
           "pixels": [[960, 540], [900, 560], [1100, 520], [700, 540], [30, 30], [960, 700]]}


def run_case(c):
    kind, m, a = c["metric"]
    metric = Schw(m) if kind == "schw" else Kerr(m, a)
    S = {"integ": c["integ"], "max_steps": c["max_steps"], "disk": c["disk"], "sky": c["sky"],
         "sky_seed": c["sky_seed"]}
    rays = []
    for px, py in c["pixels"]:
        u = (px + 0.5) / c["w"] * 2.0 - 1.0
        v = 1.0 - (py + 0.5) / c["h"] * 2.0
        st = from_camera(metric, c["cam"], u, v)
        r = trace(metric, S, c["cam"], st)
        rays.append({"px": px, "py": py, "cls": r["cls"], "attempts": r["attempts"],
                     "accepted": r["accepted"], "x": r["x"], "v": r["v"],
                     "lam": r["lam"], "intensity": r["intensity"], "rgb": r["rgb"]})
    return rays


def main():
    out = []
    for c in cases():
        out.append({"case": {k: c[k] for k in c if k != "pixels"}, "rays": run_case(c)})
    OUT.write_text(json.dumps(out, indent=1))
    print(f"wrote {OUT}")


if __name__ == "__main__":
    main()
