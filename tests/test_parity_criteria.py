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
