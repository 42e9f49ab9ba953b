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


def attempt_flops(metric_kind: str, rtol: float, stepper: int = 0) -> int:
    table = DP45_ATTEMPT_FLOPS if stepper == 1 else REFERENCE_ATTEMPT_FLOPS
    return table[(metric_kind, "rtol" if rtol > 0.0 else "tol")]
