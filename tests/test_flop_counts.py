"""The per-attempt FLOP constants used by bench.py's roofline are the oracle's
counted numbers (gargantua_b200/flops.py)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from gargantua_b200 import flops
from gargantua_b200.gr_core import Kerr, RK45Integrator, Schwarzschild


@pytest.mark.parametrize("stepper", [0, 1])
@pytest.mark.parametrize("metric_kind,mode", sorted(flops.REFERENCE_ATTEMPT_FLOPS))
def test_attempt_flops_match_oracle_count(oracle_mod, metric_kind, mode, stepper):
    L = oracle_mod.lib()
    metric = Kerr(1.0, 0.9) if metric_kind == "kerr" else Schwarzschild(1.0)
    integ = RK45Integrator(max_radius=200.0, rtol=1e-8 if mode == "rtol" else 0.0,
                           atol=1e-10 if mode == "rtol" else 0.0, stepper=stepper).to_c(10000)
    m = metric.to_c()
    st = np.array([0.0, 20.0, 1.2, 0.3, 1.3, -0.8, 0.01, 0.002, 0.0])
    out = np.zeros(10, np.uint64)
    assert L.ggo_count_attempt_ops(C.byref(m), C.byref(integ), st.ctypes.data_as(C.c_void_p),
                                   0.05, out.ctypes.data_as(C.c_void_p)) == 0
    counted = int(out[:9].sum())  # every arithmetic op and library call
    assert counted == flops.attempt_flops(metric_kind, 1e-8 if mode == "rtol" else 0.0, stepper)


@pytest.mark.parametrize("stepper", [0, 1])
@pytest.mark.parametrize("metric_kind,mode", sorted(flops.REFERENCE_ATTEMPT_FLOPS))
def test_reduced_flops_match_oracle_count(oracle_mod, metric_kind, mode, stepper):
    """The kernels' formulation, counted on the oracle built with it."""
    L = oracle_mod.lib("alt")
    metric = Kerr(1.0, 0.9) if metric_kind == "kerr" else Schwarzschild(1.0)
    rtol = 1e-8 if mode == "rtol" else 0.0
    integ = RK45Integrator(max_radius=200.0, rtol=rtol, atol=1e-10 if mode == "rtol" else 0.0,
                           stepper=stepper).to_c(10000)
    m = metric.to_c()
    st = np.array([0.0, 20.0, 1.2, 0.3, 1.3, -0.8, 0.01, 0.002, 0.0])
    out = np.zeros(10, np.uint64)
    assert L.ggo_count_attempt_ops(C.byref(m), C.byref(integ), st.ctypes.data_as(C.c_void_p),
                                   0.05, out.ctypes.data_as(C.c_void_p)) == 0
    assert int(out[:9].sum()) == flops.reduced_attempt_flops(metric_kind, rtol, stepper)
