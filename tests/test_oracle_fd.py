"""Finite-difference checks of the FP64 oracle, in the manner of test/itkFiniteDifferenceTest.cpp.

GetValue must equal GetValueAndDerivative's value exactly (itkFiniteDifferenceTest.cpp:188-217),
and central differences on parameter indices (resampling off) must match the analytic
derivative.  Control-point values are small enough that no sample crosses the moving image's
inside test while the differences are taken (that test makes the metric discontinuous).

The reference's LCC derivative is not the exact gradient of its LCC value (each control point
only collects the samples of its own support box, LCC.cu:236-244, and omits w_i), so for LCC the
check is looser and documents the size of that approximation.
"""
import numpy as np
import pytest

from helpers import make_problem
from oracle import oracle as O
from skmimageregistration_b200 import abi
from skmimageregistration_b200.abi import MetricDesc


def _fd(orc, m, params, cpw, idx, h):
    out = []
    for p in idx:
        q = params.copy()
        q[p] += h
        fp = orc.metric(m, q, cpw, derivative=False)[0]["value"]
        q[p] -= 2 * h
        fm = orc.metric(m, q, cpw, derivative=False)[0]["value"]
        out.append((fp - fm) / (2 * h))
    return np.array(out)


def _indices(g, rng, n=16):
    big = list(np.argsort(-np.abs(g))[: n // 2])
    return np.array(big + list(rng.integers(0, g.size, n // 2)))


@pytest.mark.parametrize("D", [2, 3])
@pytest.mark.parametrize("metric,regs", [
    ("mse", dict()),
    ("ncc", dict()),
    ("ncc", dict(rkhs=0.05, rd=0.05)),
    ("mse", dict(pg=0.05, pg_scaling=0.7, l2=1e-3)),
])
def test_oracle_gradient_matches_central_differences(D, metric, regs):
    shape = (10, 11, 12) if D == 3 else (22, 24)
    # unit control-point weights (the reference default): the regularizer gradients of
    # Regularizers.cu are exact gradients of their values only for w == 1
    pb, cp, cpw = make_problem(D, shape=shape, seed=7, sigma_c4=3.5, sigma_c0=7.0, cp_spacing=1.5,
                               alpha_scale=0.1, weights=False)
    orc = O.Oracle(pb)
    params = np.ascontiguousarray(cp.T.reshape(-1))
    m = MetricDesc.make(metric, use_negative_gradient=False, do_resampling=False, **regs)
    v, g = orc.metric(m, params, cpw)
    v2, _ = orc.metric(m, params, cpw, derivative=False)
    assert v["value"] == v2["value"]
    rng = np.random.default_rng(3)
    idx = _indices(g, rng)
    fd = _fd(orc, m, params, cpw, idx, 1e-5)
    err = np.abs(fd - g[idx]).max() / np.abs(g).max()
    assert err < 1e-5, err


@pytest.mark.parametrize("D", [2, 3])
def test_oracle_lcc_derivative_approximation(D):
    shape = (9, 10, 11) if D == 3 else (20, 22)
    pb, cp, cpw = make_problem(D, shape=shape, seed=9, sigma_c4=2.5, sigma_c0=5.0, cp_spacing=1.25,
                               nbh=1, alpha_scale=0.1, weights=False)
    orc = O.Oracle(pb)
    params = np.ascontiguousarray(cp.T.reshape(-1))
    m = MetricDesc.make("lcc", use_negative_gradient=False, do_resampling=False)
    v, g = orc.metric(m, params, cpw)
    rng = np.random.default_rng(5)
    idx = _indices(g, rng, 8)
    fd = _fd(orc, m, params, cpw, idx, 1e-5)
    rel = np.abs(fd - g[idx]).max() / np.abs(fd).max()
    # the reference's LCC derivative points the same way as the true gradient but is not equal to it
    cos = float(fd @ g[idx] / (np.linalg.norm(fd) * np.linalg.norm(g[idx])))
    print("LCC: max |fd - g| / max |fd| = %.3f, cosine = %.3f" % (rel, cos))
    assert cos > 0.5
