"""Multi-scale driver: FP64 restatements of the preprocessing and the configuration semantics (CPU)."""
import numpy as np
import pytest

from oracle import multiscale as M
from skmimageregistration_b200 import abi
from skmimageregistration_b200.register import DEFAULT_CONFIG, current, make_desc


def test_gaussian_kernel_is_a_normalised_discrete_gaussian():
    for t in (0.25, 1.0, 2.0, 7.5):
        c = M.gaussian_half_kernel(t)
        assert abs(c[0] + 2 * c[1:].sum() - 1.0) < 1e-14
        assert np.all(np.diff(c) < 0)                      # decreasing away from the centre
        # variance of the discrete Gaussian e^-t I_n(t) is t; truncation at 1% of the mass lowers it
        n = np.arange(len(c))
        var = 2 * (c * n * n).sum()
        assert 0.8 * t < var <= t * 1.000001


def test_gaussian_kernel_width_limit():
    c = M.gaussian_half_kernel(5000.0, 0.01, 64)
    assert len(c) == 65                                    # stops once the half kernel exceeds 64 entries
    assert abs(c[0] + 2 * c[1:].sum() - 1.0) < 1e-14


def test_smoothing_keeps_constants_and_mass_away_from_borders():
    img = np.full((9, 11, 13), 3.25)
    out = M.gaussian_smooth(img, (1.0, 2.0, 0.5), 2.0)
    assert np.allclose(out, 3.25, rtol=0, atol=1e-13)
    spike = np.zeros((31, 33))
    spike[15, 16] = 1.0
    out = M.gaussian_smooth(spike, (1.0, 1.0), 1.5)
    assert abs(out.sum() - 1.0) < 1e-13                   # kernel inside the image: mass preserved
    # separable: the 2-D response is the outer product of the two 1-D kernels
    c = M.gaussian_half_kernel(1.5)
    k = np.concatenate([c[:0:-1], c])
    r = len(c) - 1
    assert np.allclose(out[15 - r:16 + r, 16 - r:17 + r], np.outer(k, k), atol=1e-15)


def test_threshold_rescale_semantics():
    v = np.array([[-2000.0, -5.0, 0.0], [10.0, 3400.0, 4000.0]])
    out = M.threshold_rescale(v, (-1500, 3500))
    # clamp to [smallest value above -1500, largest below 3500] = [-5, 3400], then onto [0, 1]
    ref = (np.clip(v, -5.0, 3400.0) + 5.0) / 3405.0
    assert np.allclose(out, ref, rtol=0, atol=1e-15)
    out = M.threshold_rescale(v, None)
    assert np.allclose(out, (v + 2000.0) / 6000.0, atol=1e-15)
    with pytest.raises(ValueError):
        M.threshold_rescale(np.array([5000.0, 6000.0]), (-1500, 3500))


def test_current_repeats_the_last_entry():
    c = dict(DEFAULT_CONFIG, sigma_C4=[32, 16], num_scales=4)
    assert [current(c, "sigma_C4", s) for s in range(4)] == [32, 16, 16, 16]
    assert current(c, "cp_spacing_scaler", 3) == 4.0
    d = make_desc(dict(c, metric="ncc"), 3)
    assert d.num_scales == 4 and d.metric == abi.NCC
    assert list(d.sigma_c4[:4]) == [32.0, 16.0, 16.0, 16.0]
    assert list(d.sampling_rate[:4]) == [5, 4, 3, 3]
    assert d.apply_threshold == 1 and d.threshold_min == -1500 and d.threshold_max == 3500
    with pytest.raises(ValueError):
        make_desc(dict(c, tensor_weights=[400]), 3)
