"""Algorithmic floating-point work of one RK45 attempt.

Counted, not estimated: the CPU oracle's metric and stepper templates run one
accepted attempt over a counting double that tallies every +, -, *, /, unary
minus, sqrt, sin, cos, pow and exp (each counts one FLOP).  This is the work
the reference does per attempt, including Kerr's dense 64-entry Christoffel
contraction (crates/gr-core/src/metric.rs:37-52).  tests/test_flop_counts.py
re-counts them on the oracle and fails if they drift.
"""
from __future__ import annotations

# (metric, error-norm mode) -> FLOPs per attempt of the reference formulation
REFERENCE_ATTEMPT_FLOPS = {
    ("kerr", "rtol"): 2801,
    ("kerr", "tol"): 2787,
    ("schwarzschild", "rtol"): 673,
    ("schwarzschild", "tol"): 659,
}


# The same count for one attempt of the full Dormand-Prince stepper
# (abi.GG_STEPPER_DP45): the seven right-hand sides and the stage algebra
# of all eight components, as the oracle's step_dp45 restates it.
DP45_ATTEMPT_FLOPS = {
    ("kerr", "rtol"): 3084,
    ("kerr", "tol"): 3078,
    ("schwarzschild", "rtol"): 956,
    ("schwarzschild", "tol"): 950,
}


# What the kernels compute instead: Kerr's right-hand side from its ~20
# non-zero Christoffel symbols in closed form (one reciprocal, shared
# subexpressions) rather than the dense 64-entry contraction, counted the
# same way on the oracle's build with that arrangement (liboracle_gg_alt.so).
# Schwarzschild's reference RHS is already the inlined sparse form.
REDUCED_ATTEMPT_FLOPS = {
    (("kerr", "rtol"), 0): 1394,
    (("kerr", "tol"), 0): 1380,
    (("kerr", "rtol"), 1): 1677,
    (("kerr", "tol"), 1): 1671,
}


def attempt_flops(metric_kind: str, rtol: float, stepper: int = 0) -> int:
    table = DP45_ATTEMPT_FLOPS if stepper == 1 else REFERENCE_ATTEMPT_FLOPS
    return table[(metric_kind, "rtol" if rtol > 0.0 else "tol")]


def reduced_attempt_flops(metric_kind: str, rtol: float, stepper: int = 0) -> int:
    """FLOPs per attempt of the formulation the kernels run."""
    key = (metric_kind, "rtol" if rtol > 0.0 else "tol")
    if metric_kind != "kerr":
        return attempt_flops(metric_kind, rtol, stepper)
    return REDUCED_ATTEMPT_FLOPS[(key, 1 if stepper == 1 else 0)]
