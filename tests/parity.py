"""Parity criteria of the FP64 form against the CPU oracle (shared by the GPU
parity tests and by tests/test_parity_criteria.py, which checks on the CPU
that the criteria reject planted mistakes)."""
from __future__ import annotations

import numpy as np

from gargantua_b200.accuracy import crossing_geo_err  # noqa: F401  (re-exported)
from gargantua_b200.curved import Scene

TWO_PI = 2.0 * np.pi
REL = 1e-9  # endpoint tolerance of the FP64 form


def rel_err(a: np.ndarray, b: np.ndarray, angle_row: int | None = 3) -> np.ndarray:
    d = a - b
    if angle_row is not None:
        d[angle_row] = np.remainder(d[angle_row] + np.pi, TWO_PI) - np.pi
    scale = np.maximum(np.abs(b).max(axis=0), 1e-300)
    return np.abs(d).max(axis=0) / scale


def endpoint_err(scene: Scene, x, v, o) -> np.ndarray:
    """Relative endpoint difference of (x, v) against oracle outputs o.  Rays
    that end at the horizon are compared on (r, theta) only: t, phi and the
    velocity diverge there in Boyer-Lindquist coordinates."""
    e = np.maximum(rel_err(x.copy(), o.x.copy()), rel_err(v.copy(), o.v.copy(), angle_row=None))
    rh = scene.metric.event_horizon() or 0.0
    at_h = o.x[1] < rh + scene.integrator_c().horizon_buffer + 1e-12
    e[at_h] = (np.abs(x[1:3, at_h] - o.x[1:3, at_h]) /
               np.abs(o.x[1:3, at_h]).max(axis=0)).max(axis=0)
    return e


def compare(scene: Scene, g, o, oracle_mod, idx=None, max_excluded=0.005):
    """Compares GPU outputs g with oracle outputs o (index arrays aligned).

    The reference algorithm is itself ill-conditioned on some rays: its
    step-size law divides by an error estimate that cancels to ~tol, and
    strong-field / photon-ring trajectories amplify any last-bit change.  The
    size of that effect is measured on the CPU by tracing the same samples
    through two builds of the oracle that round differently: one with fused
    multiply-adds, one with Kerr's right-hand side in an algebraically
    equivalent arrangement (oracle/Makefile).  The GPU must then be no worse
    than that: at every threshold t in 1e-9 .. 1e-6, the number of samples
    whose endpoint differs from the oracle's by more than t is at most twice
    the FMA build's count (plus 0.1 % of the samples).  Per sample, only
    gross outliers are tested: a difference beyond max(1e-5, 100 x the larger
    of its two measured sensitivities), or a different class, must lie
    within 1e-6 M of a class boundary.  (Two independent roundings of an
    ill-conditioned ray differ by heavy-tailed ratios, so tighter per-sample
    bounds test chance, not the kernel; the amplified rounding tops out near
    3e-6 at a = 0.998, while a stepping or crossing error shows as 1e-3.)
    """
    idx = np.arange(len(o.cls)) if idx is None else np.asarray(idx)
    sub = len(g.cls) != len(o.cls)
    sel = idx if sub else slice(None)
    gc = g.cls[sel]
    same = gc == o.cls
    e_gpu = endpoint_err(scene, g.x[:, sel], g.v[:, sel], o)
    sens = {}
    for variant in ("fma", "alt"):
        f = oracle_mod.trace_samples(scene, idx.astype(np.uint64), variant=variant)
        e = endpoint_err(scene, f.x, f.v, o)
        e[f.cls != o.cls] = np.inf
        sens[variant] = e
    e_fma = sens["fma"]
    e_sens = np.maximum(sens["fma"], sens["alt"])
    n = len(o.cls)
    slack = max(3, int(0.001 * n))
    for t in (1e-9, 1e-8, 1e-7, 1e-6):
        ng = int((same & (e_gpu > t)).sum())
        nf = int((e_fma > t).sum())
        assert ng <= 2 * nf + slack, f"{ng} samples beyond {t:g} on the GPU vs {nf} for the FMA build"
    suspects = np.nonzero(~same | (e_gpu > np.maximum(1e-5, 100.0 * e_sens)))[0]
    assert len(suspects) <= max(3, max_excluded * n), f"{len(suspects)} samples differ"
    for k in suspects:
        assert oracle_mod.near_class_boundary(scene, int(idx[k])), (
            f"sample {idx[k]} (class {gc[k]} vs {o.cls[k]}, endpoint rel {e_gpu[k]:.2e}, "
            f"rounding sensitivity {e_sens[k]:.2e}) differs away from any class boundary")
    ga = g.attempts[sel]
    att_same = (ga == o.attempts)[same].mean()
    assert att_same > 0.999, att_same
    strict = (e_gpu[same] <= REL).mean()
    return {"class_mismatch": int((~same).sum()), "excluded": int(len(suspects)),
            "within_1e-9": float(strict), "attempts_equal": float(att_same)}



def fp32_amplification(scene, oracle_mod, index: int, ref_cross: np.ndarray,
                       delta: float = 1e-7) -> float:
    """How much the FP64 oracle amplifies an input perturbation at the FP32
    rounding level: sample `index` re-shot with its image-plane point moved by
    `delta` in u and in v, crossing-state change (crossing_geo_err against
    ref_cross, the unperturbed crossing) over delta, the larger of the two.
    A ray whose amplification is well above 1 cannot hold 1e-6 in any FP32
    representation of its state; infinite when the perturbed ray ends
    elsewhere."""
    from gargantua_b200.accuracy import crossing_geo_err as geo
    u, v = oracle_mod.sample_uv(scene, int(index))
    worst = 0.0
    for du, dv in ((delta, 0.0), (0.0, delta)):
        c = np.asarray(oracle_mod.trace_uv(scene, u + du, v + dv).cross).reshape(8, 1)
        if not np.isfinite(c[0, 0]):
            return float("inf")
        worst = max(worst, float(geo(c, ref_cross.reshape(8, 1))[0]) / delta)
    return worst


def mixed_report(scene, g_cross, o_cross, oracle_mod, index=None, tol=1e-6,
                 min_amplification=3.0, delta=1e-7):
    """Crossing-state error of a mixed-precision render against the oracle's
    FP64 crossings.  For every ray beyond `tol` the oracle's amplification of
    an FP32-sized (`delta`) perturbation is measured: rays it amplifies by at
    most `min_amplification` are the mixed form's own failures
    ("unexplained"); for the rest, "worst_ratio" is the largest error over
    amplification x delta, the error the oracle itself shows from such a
    perturbation (1 = as large)."""
    index = np.arange(g_cross.shape[1]) if index is None else np.asarray(index)
    m = np.isfinite(o_cross[0]) & np.isfinite(g_cross[0])
    e = crossing_geo_err(g_cross[:, m], o_cross[:, m])
    over = np.nonzero(e > tol)[0]
    unexplained, ratios = [], []
    for k in over:
        amp = fp32_amplification(scene, oracle_mod, index[m][k], o_cross[:, m][:, k], delta)
        if amp <= min_amplification:
            unexplained.append(int(index[m][k]))
        elif np.isfinite(amp):
            ratios.append(float(e[k]) / (amp * delta))
    return {"rays": int(m.sum()), "p50": float(np.quantile(e, 0.5)),
            "p99": float(np.quantile(e, 0.99)), "p99.9": float(np.quantile(e, 0.999)),
            "max": float(e.max()), "over_tol": int(over.size), "unexplained": unexplained,
            "worst_ratio": max(ratios) if ratios else 0.0}
