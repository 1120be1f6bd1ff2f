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
    assert list(d.tensor_weights[:4]) == [400.0, 200.0, 100.0, 100.0]   # the reference's defaults
    d = make_desc(dict(c, tensor_weights=[0]), 3)
    assert list(d.tensor_weights[:4]) == [0.0] * 4
    assert not d.guidance_image and not d.weight_tensor and not d.weight_image


# --- anisotropic covariance tensor (include/AnisotropicTensorUtils.h) ------------------------

def test_image_gradient_central_differences_with_repeated_edges():
    f = np.array([[0.0, 1.0, 4.0, 9.0]])                  # one row, x = 0..3
    g = M.image_gradient(f, (0.5, 1.0))
    assert np.allclose(g[0, :, 0], [(1 - 0) / 1.0, (4 - 0) / 1.0, (9 - 1) / 1.0, (9 - 4) / 1.0])
    assert np.allclose(g[..., 1], 0.0)                    # a single row: y neighbours are the texel itself


def _cov_known(lams, D, align):
    """Covariance the reference builds for a diagonal structure tensor diag(lams)."""
    order = np.argsort(np.abs(lams), kind="stable")
    main = order[-1]
    n = np.zeros(D)
    n[main] = 1.0
    lam = abs(lams[main])
    if 0 <= align < D:
        m = np.zeros(D)
        m[align] = 1.0
        cr = abs(n[0] * m[1] - n[1] * m[0]) if D == 2 else np.linalg.norm(np.cross(n, m))
        lam *= (cr + 1e-10) ** 2 / np.sqrt(D)
    p = lam ** 1.5
    cov = np.diag([1.0 + p / (1.0 + p)] * D)
    cov[main, main] = 1.0 / (1.0 + p)
    return cov, lam


@pytest.mark.parametrize("lams,align", [((4.0, 1.0), 2), ((1.0, 4.0), 2), ((4.0, 1.0), 1), ((9.0, 4.0, 1.0), 2),
                                        ((1.0, 9.0, 4.0), 2), ((1.0, 4.0, 9.0), 2), ((9.0, 4.0, 1.0), 0),
                                        ((2.0, 3.0, 5.0), -1)])
def test_covariance_known_answers_on_diagonal_tensors(lams, align):
    D = len(lams)
    cov, tilt, bad = M.covariance_from_structure(np.diag(lams)[None], align)
    ref, lam = _cov_known(np.asarray(lams), D, align)
    assert bad == 0
    assert np.allclose(cov[0], ref, rtol=0, atol=1e-14)
    assert abs(tilt - lam) <= 1e-14 * max(1.0, lam)


def test_covariance_identity_where_an_eigenvalue_vanishes():
    T = np.zeros((3, 3, 3))
    T[0] = np.diag([5.0, 2.0, 0.0])                       # rank 2
    T[1] = np.diag([5.0, 2.0, 5e-9])                      # below the 1e-8 test
    T[2] = np.diag([5.0, 2.0, 2e-8])                      # passes
    cov, tilt, bad = M.covariance_from_structure(T, 2)
    assert np.allclose(cov[0], np.eye(3)) and np.allclose(cov[1], np.eye(3))
    assert not np.allclose(cov[2], np.eye(3))
    _, none, _ = M.covariance_from_structure(np.zeros((2, 2, 2)), 2)
    assert none == -np.finfo(np.float64).max


def test_covariance_rotates_with_the_structure_tensor_in_2d():
    rng = np.random.default_rng(4)
    A = rng.normal(size=(50, 2, 2))
    T = A @ A.transpose(0, 2, 1) + 0.1 * np.eye(2)
    th = 0.7
    R = np.array([[np.cos(th), -np.sin(th)], [np.sin(th), np.cos(th)]])
    cov, _, _ = M.covariance_from_structure(T, -1)
    cov_r, _, _ = M.covariance_from_structure(R @ T @ R.T, -1)
    assert np.allclose(cov_r, R @ cov @ R.T, atol=1e-12)
    ev = np.linalg.eigvalsh(cov)
    assert ev.min() > 0 and ev.max() < 2                  # 1/(1+p) and 1 + p/(1+p)


def test_anisotropic_tensor_constant_and_ramp_images_give_identity():
    for img in (np.full((9, 10, 11), 0.7), np.broadcast_to(np.arange(11.0), (9, 10, 11))):
        cov, tilt = M.anisotropic_tensor(img, (1.0, 1.0, 1.0), 8.0, 400.0, 2)
        assert np.allclose(cov, np.eye(3), atol=1e-12)       # rank <= 1 structure: identity
        assert tilt == -np.finfo(np.float64).max
