"""The mixed form's step-size factor on the squared error norm.

An accepted attempt's step grows by 0.9 (tol / err)^(1/5) (the reference's
law, geodesic.rs:310-321).  The mixed attempt forms err^2 = s2 / 8 in FP64
and takes the factor as (8 / s2)^(1/10) directly: a seed from the FP32 power
and two Newton steps, with s2 scaled by 1e30 below 8e-30 so that the FP32
seed does not underflow, and s2 taken as 8e-60 below that (a factor of 1e6,
as the FP64 form's clamp of tol / err at 1e30).  Checked here against the
closed form in numpy on 200,000 values from 1e-70 to 8, and at the branch
edges.  The bar is exact: w^10 s2 / 8 in rational arithmetic, since numpy's
pow(x, 0.1) carries the binary 0.1's own error."""
from __future__ import annotations

import ctypes as C
from fractions import Fraction

import numpy as np
import pytest

from gargantua_b200 import abi


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    return torch


@pytest.mark.gpu
def test_step_factor_matches_closed_form(torch_cuda, gglib):
    rng = np.random.default_rng(5)
    s2 = np.concatenate([10.0 ** rng.uniform(-70.0, np.log10(8.0), 200_000),
                         [8e-60, 8e-60 * (1 + 1e-15), 8e-30, 8e-30 * (1 - 1e-15), 7.999999, 1.0,
                          1e-300, 5e-324]])
    x = torch_cuda.from_numpy(s2).cuda()
    out = torch_cuda.empty_like(x)
    st = gglib.gg_check_step_factor(C.c_void_p(x.data_ptr()), C.c_void_p(out.data_ptr()), len(s2),
                                    None)
    assert st == abi.GG_OK
    got = out.cpu().numpy()
    assert np.isfinite(got).all()
    clamped = np.maximum(s2, 8e-60)
    # against the closed form: pow's exponent 0.1 is not 1/10 in binary, which
    # alone moves x^0.1 by 5.5e-18 ln x (7e-16 at x = 1e58), so the bar here is
    # loose and the exact check follows
    want = (8.0 / clamped) ** 0.1
    assert (np.abs(got - want) / want).max() < 2e-15
    # exactly, in rational arithmetic on the doubles: w^10 s2 / 8 = 1 + 10 e
    # for a relative error e of w
    idx = np.concatenate([np.arange(len(s2) - 8, len(s2)),
                          np.random.default_rng(6).choice(len(s2) - 8, 3000, replace=False)])
    worst = 0.0
    for i in idx:
        r = Fraction(float(got[i])) ** 10 * Fraction(float(clamped[i])) / 8 - 1
        worst = max(worst, abs(float(r)) / 10.0)
    assert worst < 6e-16, worst  # measured 3.8e-16: about 2 ulp
    assert got[s2 <= 8e-60].max() == pytest.approx(1e6, rel=1e-15)


@pytest.mark.gpu
def test_step_factor_rejects_null(torch_cuda, gglib):
    assert gglib.gg_check_step_factor(None, None, 0, None) == abi.GG_OK
    assert gglib.gg_check_step_factor(None, None, 4, None) == abi.GG_ERR_INVALID_ARG
