"""The vector-Jacobian product of one Kerr right-hand side, which the
differentiable render's backward takes at every Dormand-Prince stage.

The device has it in two forms (gg_vjp.cuh): dual numbers run through the
templated physics, and a hand-written reverse pass that the backward uses.
Both are checked here on the same points: against each other to rounding,
and against central differences of the oracle's geodesic acceleration
(the reference's dense Christoffel contraction, metric.rs:37-52), which
shares no code with either."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from gargantua_b200 import abi
from gargantua_b200.gr_core import Kerr

PI = np.pi


def random_points(n: int, seed: int) -> np.ndarray:
    """n rows of (M, a, r, theta, w[4], kb[4]) outside the horizon and away
    from the poles, as the backward meets them."""
    rng = np.random.default_rng(seed)
    q = np.empty((n, 12))
    q[:, 0] = 1.0
    q[:, 1] = rng.uniform(-0.998, 0.998, n)
    rh = 1.0 + np.sqrt(1.0 - q[:, 1] ** 2)
    q[:, 2] = rh + 0.05 + rng.uniform(0.0, 1.0, n) ** 2 * 200.0
    q[:, 3] = rng.uniform(0.02, PI - 0.02, n)
    q[:, 4:8] = rng.normal(size=(n, 4))
    q[:, 8:12] = rng.normal(size=(n, 4))
    return q


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    return torch


def device_vjp(torch, gglib, q: np.ndarray, form: int) -> np.ndarray:
    qd = torch.from_numpy(np.ascontiguousarray(q)).cuda()
    out = torch.full((len(q), 7), np.nan, dtype=torch.float64, device="cuda")
    st = gglib.gg_check_kerr_vjp(C.c_void_p(qd.data_ptr()), C.c_void_p(out.data_ptr()),
                                 len(q), form, None)
    assert st == abi.GG_OK
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.gpu
def test_check_entry_rejects_bad_arguments(torch_cuda, gglib):
    x = torch_cuda.zeros(24, dtype=torch_cuda.float64, device="cuda")
    p = C.c_void_p(x.data_ptr())
    assert gglib.gg_check_kerr_vjp(None, p, 1, 0, None) == abi.GG_ERR_INVALID_ARG
    assert gglib.gg_check_kerr_vjp(p, p, 1, 2, None) == abi.GG_ERR_INVALID_ARG
    assert gglib.gg_check_kerr_vjp(None, None, 0, 0, None) == abi.GG_OK


@pytest.mark.gpu
def test_hand_reverse_pass_equals_dual_numbers(torch_cuda, gglib):
    q = random_points(200_000, 11)
    hand = device_vjp(torch_cuda, gglib, q, 0)
    dual = device_vjp(torch_cuda, gglib, q, 1)
    assert np.isfinite(hand).all() and np.isfinite(dual).all()
    # per point, relative to the largest of its seven products
    scale = np.abs(dual).max(axis=1, keepdims=True)
    rel = np.abs(hand - dual) / scale
    assert rel.max() < 1e-11, (rel.max(), q[rel.max(axis=1).argmax()])


@pytest.mark.gpu
def test_hand_reverse_pass_matches_oracle_differences(torch_cuda, gglib, oracle_mod):
    """Fourth-order central differences of kb . a(x, w; spin) through the
    oracle's dense contraction.  The steps are 1e-3 of the distance to what
    the products blow up at: the horizon for r (r - r_+) and for the spin
    (Delta, through which a moves the horizon), the nearer pole for theta.
    That keeps the truncation near 1e-12 even at r_+ + 0.05; the bar, 1e-8 of
    the product's scale, leaves the differences' rounding room."""
    q = random_points(400, 12)
    hand = device_vjp(torch_cuda, gglib, q, 0)
    lib = oracle_mod.lib()

    def kb_dot_a(row: np.ndarray) -> float:
        m = Kerr(row[0], row[1]).to_c()
        pos = np.array([0.0, row[2], row[3], 0.0])
        vel = np.ascontiguousarray(row[4:8])
        a = np.zeros(4)
        lib.ggo_geodesic_acceleration(C.byref(m), oracle_mod._ptr(pos), oracle_mod._ptr(vel),
                                      oracle_mod._ptr(a))
        return float(row[8:12] @ a)

    # output column -> input column of the point row
    cols = {0: 2, 1: 3, 2: 4, 3: 5, 4: 6, 5: 7, 6: 1}
    worst = 0.0
    for i, row in enumerate(q):
        m_, a_, r_, th_ = row[:4]
        step = {2: 1e-3 * (r_ - (m_ + np.sqrt(m_ * m_ - a_ * a_))),
                3: 1e-3 * min(th_, PI - th_),
                1: 1e-3 * min(1.0, r_ * r_ - 2.0 * m_ * r_ + a_ * a_)}
        for out_c, in_c in cols.items():
            h = step.get(in_c, 1e-3)

            def f(e: float) -> float:
                x = row.copy()
                x[in_c] += e
                return kb_dot_a(x)

            fd = (8.0 * (f(h) - f(-h)) - (f(2 * h) - f(-2 * h))) / (12.0 * h)
            err = abs(hand[i, out_c] - fd) / max(abs(fd), 1e-3 * np.abs(hand[i]).max(), 1e-12)
            worst = max(worst, err)
    assert worst < 1e-8, worst
