"""The box-window LCC oracle (oracle/lcc_box.py) pinned without a reference implementation.

No reference code computes the box-window LCC, so its restatement is checked by its own
properties: the separable box sum against a direct loop, invariance of the value under affine
intensity changes of either image, and the derivative against FP64 central differences of the
value in the manner of itkFiniteDifferenceTest.
"""
import itertools

import numpy as np
import pytest

from helpers import make_problem
from oracle import lcc_box as LB


def test_box_sum_matches_a_direct_loop():
    rng = np.random.default_rng(0)
    a = rng.normal(size=(5, 7, 9))
    out = LB.box_sum(a)
    ref = np.zeros_like(a)
    for z, y, x in itertools.product(range(5), range(7), range(9)):
        ref[z, y, x] = a[max(z - 2, 0):z + 3, max(y - 2, 0):y + 3, max(x - 2, 0):x + 3].sum()
    np.testing.assert_allclose(out, ref, rtol=0, atol=1e-12)


@pytest.mark.parametrize("D", [2, 3])
def test_value_is_invariant_under_affine_intensity_changes(D):
    rng = np.random.default_rng(1)
    shape = (12, 13, 14)[:D] if D == 3 else (20, 23)
    f = rng.uniform(0, 1, shape)
    m = 0.5 * f + rng.normal(0, 0.1, shape)
    valid = rng.uniform(0, 1, shape) > 0.1
    v0, n0, _ = LB.window_terms(f, m, valid)
    v1, n1, _ = LB.window_terms(3.0 * f - 7.0, -0.25 * m + 2.0, valid)
    assert n0 == n1 > 0
    assert abs(v1 - v0) <= 1e-10 * abs(v0)
    assert -1.0 <= v0 < 0.0


def test_flat_windows_are_not_counted():
    f = np.ones((9, 9, 9))
    m = np.linspace(0, 1, 729).reshape(9, 9, 9)
    v, n, coef = LB.window_terms(f, m, np.ones(f.shape, bool))
    assert n == 0 and v == 0.0 and not np.any(coef)


@pytest.mark.parametrize("D", [2, 3])
def test_derivative_matches_central_differences(D):
    shape = (12, 13, 14) if D == 3 else (26, 28)
    pb, cp, cpw = make_problem(D, shape=shape, seed=3, sigma_c4=4.5, sigma_c0=9.0, cp_spacing=2.5)
    val, count, der = LB.evaluate(pb, cp, cpw)
    assert count > 0 and -1.0 <= val < 0.0
    gmax = np.abs(der).max()
    assert gmax > 0
    C = pb.C
    h = 1e-4
    for i in np.argsort(-np.abs(der))[:8]:
        d, j = divmod(int(i), C)
        cpp, cpm = cp.copy(), cp.copy()
        cpp[j, d] += h
        cpm[j, d] -= h
        vp, np_, _ = LB.evaluate(pb, cpp, cpw, derivative=False)
        vm, nm, _ = LB.evaluate(pb, cpm, cpw, derivative=False)
        assert np_ == nm == count
        fd = (vp - vm) / (2 * h)
        assert abs(fd - der[i]) <= 1e-5 * gmax, (i, fd, der[i])
