"""The GPU parity criteria (tests/parity.py) checked on the CPU: they accept a
differently rounded run of the reference algorithm and reject planted
mistakes.  The stand-in "GPU" outputs are the oracle's own (FMA build =
rounding change only); the mistakes are planted in copies of those outputs."""
from __future__ import annotations

import copy

import numpy as np
import pytest

from gargantua_b200 import workloads
from parity import compare


@pytest.fixture(scope="module")
def runs(oracle_mod):
    scene = workloads.schwarzschild_thin_256()
    scene.width = scene.height = 96
    _, o = oracle_mod.render(scene)
    _, f = oracle_mod.render(scene, variant="fma")
    return scene, o, f


def test_rounding_change_passes(oracle_mod, runs):
    scene, o, f = runs
    rep = compare(scene, f, o, oracle_mod)
    assert rep["class_mismatch"] == 0 and rep["within_1e-9"] > 0.999


def test_planted_endpoint_error_is_caught(oracle_mod, runs):
    scene, o, f = runs
    bad = copy.deepcopy(f)
    esc = np.nonzero(bad.cls == 1)[0][::50]
    bad.x[1, esc] *= 1.0 + 1e-4  # r off by 1e-4 on 2 % of the escaped rays
    with pytest.raises(AssertionError):
        compare(scene, bad, o, oracle_mod)


def test_planted_class_flip_is_caught(oracle_mod, runs):
    scene, o, f = runs
    bad = copy.deepcopy(f)
    far = np.nonzero(bad.cls == 1)[0][len(bad.cls) // 4]  # an escaped ray mid-sky
    bad.cls[far] = 0
    with pytest.raises(AssertionError, match="away from any class boundary"):
        compare(scene, bad, o, oracle_mod)


def test_planted_step_count_error_is_caught(oracle_mod, runs):
    scene, o, f = runs
    bad = copy.deepcopy(f)
    bad.attempts[::100] += 1
    with pytest.raises(AssertionError):
        compare(scene, bad, o, oracle_mod)


# ---- the mixed form's criterion (tests/test_mixed.py) ------------------------------
def _dp45_subset(oracle_mod):
    from gargantua_b200 import abi
    scene = workloads.schwarzschild_thin_256(stepper=abi.GG_STEPPER_DP45)
    idx = np.arange(0, scene.n_samples, 997, dtype=np.uint64)
    return scene, idx, oracle_mod.trace_cross(scene, idx)


def test_mixed_criterion_accepts_fp32_sized_noise(oracle_mod):
    from parity import mixed_report
    scene, idx, oc = _dp45_subset(oracle_mod)
    noisy = oc * (1.0 + 3e-8 * np.random.default_rng(0).standard_normal(oc.shape))
    rep = mixed_report(scene, noisy, oc, oracle_mod, index=idx)
    assert rep["p99"] <= 1e-6 and rep["unexplained"] == []


def test_mixed_criterion_flags_error_on_well_conditioned_rays(oracle_mod):
    """A 5e-6 error planted in the radius of well-conditioned rays is not
    excused as ill-conditioning."""
    from parity import mixed_report
    scene, idx, oc = _dp45_subset(oracle_mod)
    bad = oc.copy()
    bad[1, :5] *= 1.0 + 5e-6
    rep = mixed_report(scene, bad, oc, oracle_mod, index=idx)
    assert len(rep["unexplained"]) >= 4
