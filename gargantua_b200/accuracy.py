"""Accuracy measures of a render against a reference render of the same samples."""
from __future__ import annotations

import numpy as np


def crossing_geo_err(c: np.ndarray, ref: np.ndarray) -> np.ndarray:
    """Per-ray error of a crossing state c (8 x n: t, r, theta, phi and their
    derivatives) against ref, measured geometrically so that angles are not
    judged against r ~ 200: the Cartesian position difference over r, the
    Cartesian spatial-velocity difference over its length (direction and
    speed), and t and dt/dlambda relative.  The largest of the four."""
    def cart(x):
        r, th, ph = x[1], x[2], x[3]
        st, ct, sp, cp = np.sin(th), np.cos(th), np.sin(ph), np.cos(ph)
        rhat = np.stack([st * cp, st * sp, ct])
        thhat = np.stack([ct * cp, ct * sp, -st])
        phhat = np.stack([-sp, cp, np.zeros_like(sp)])
        pos = r * rhat
        vel = x[5] * rhat + r * x[6] * thhat + r * st * x[7] * phhat
        return pos, vel
    pc, vc = cart(c)
    pr, vr = cart(ref)
    e_pos = np.linalg.norm(pc - pr, axis=0) / np.linalg.norm(pr, axis=0)
    e_vel = np.linalg.norm(vc - vr, axis=0) / np.linalg.norm(vr, axis=0)
    e_t = np.abs(c[0] - ref[0]) / np.maximum(np.abs(ref[0]), 1e-300)
    e_vt = np.abs(c[4] - ref[4]) / np.abs(ref[4])
    return np.maximum.reduce([e_pos, e_vel, e_t, e_vt])
