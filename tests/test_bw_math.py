"""The FP32 integrators' Balloon-Windkessel e^y - 1 and ln(1 + x)
(fp32_model.cuh expm1_bw / log1p_bw: Taylor / Mercator series near zero,
hardware base-2 exponential and logarithm elsewhere) against CUDA's expm1f
and log1pf on the device, over the arguments the step produces: e^y - 1 of
(1/alpha) ln(nu), (1/alpha - 1) ln(nu) and -ln(1 - rho) (1/f - 1), ln(1 + x)
of nu - 1, with nu and f within [0.5, 2] (BOLD deviations stay far inside).

Bar: relative error 1e-5 (4e-5 next to the switch point, |y| = 1/16, where
subtracting 1 from the base-2 exponential magnifies its error 17 times);
the end effect on BOLD is covered by the oracle parity tests."""
import numpy as np
import pytest

import bnm_cuda_b200 as B

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.abs(a.astype(np.float64) - b) / np.maximum(np.abs(b), 1e-30)


def test_expm1_and_log1p_of_the_bw_step_match_cuda():
    rng = np.random.default_rng(3)
    lo, hi = np.log(0.5) * 3.125, np.log(2.0) * 3.125  # widest argument: (1/alpha) ln(nu)
    y = np.concatenate([rng.uniform(lo, hi, 200_000), rng.uniform(-0.07, 0.07, 100_000),
                        np.array([0.0, 1e-8, -1e-8, 0.0625, -0.0625, 0.0624999, -0.0624999])]).astype(np.float32)
    r = B.bw_math_probe(y)
    ref = np.expm1(y.astype(np.float64))
    err_e = _rel(r[:, 0], ref)
    cuda_e = _rel(r[:, 1], ref)
    near = np.abs(y) < 0.07
    assert err_e[~near].max() < 1e-5, err_e[~near].max()
    assert err_e[near].max() < 4e-5, err_e[near].max()
    assert cuda_e.max() < 1e-6  # the reference point itself
    x = np.concatenate([rng.uniform(-0.5, 1.0, 200_000), rng.uniform(-0.07, 0.07, 100_000),
                        np.array([0.0, 1e-8, -1e-8, 0.0625, -0.0625])]).astype(np.float32)
    r = B.bw_math_probe(x)
    ref = np.log1p(x.astype(np.float64))
    err_l = _rel(r[:, 2], ref)
    assert err_l.max() < 1e-5, err_l.max()
    assert _rel(r[:, 3], ref).max() < 1e-6
