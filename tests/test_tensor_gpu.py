"""Anisotropic covariance tensor (ComputeAnisotropicTensor, include/AnisotropicTensorUtils.h:37-371)
on the GPU against the FP64 restatement, and the registration driver with kernel weighting.

Tolerances:
  * tensor (FP64 on both sides, Jacobi on the GPU vs LAPACK in the oracle): max |a - b| <= 1e-9
    over the covariance entries (which lie in (0, 2)), maximum tilt relative error <= 1e-10;
  * registration: as the multi-scale driver tests (displacement 1e-3 of its maximum, per-level
    best value 1e-4 relative), the FP32 anisotropic evaluator against the FP64 oracle evaluator.
"""
import numpy as np
import pytest

from helpers import max_rel, rel_err, smooth_volume
from oracle import multiscale as M
from skmimageregistration_b200 import register as R
from skmimageregistration_b200.evaluator import SkmError

pytestmark = pytest.mark.gpu

DBL_LOWEST = -np.finfo(np.float64).max


def _image(shape, seed, noise=0.05):
    rng = np.random.default_rng(seed)
    return smooth_volume(rng, shape) + noise * rng.normal(size=shape)


@pytest.mark.parametrize("shape,spacing,sigma,weight,align", [
    ((40, 44), (1.0, 1.5), 8.0, 400.0, 2),          # 2-D: axis 2 does not exist, no alignment weighting
    ((40, 44), (1.0, 1.0), 16.0, 200.0, 1),         # 2-D aligned with y
    ((14, 16, 18), (1.0, 0.8, 1.2), 8.0, 400.0, 2),  # the form the registration driver calls
    ((14, 16, 18), (1.0, 1.0, 1.0), 32.0, 100.0, -1),
    ((12, 9, 20), (2.0, 1.0, 0.5), 4.0, 50.0, 0),
])
def test_anisotropic_tensor_matches_oracle(shape, spacing, sigma, weight, align):
    img = _image(shape, 11)
    cov, tilt = R.anisotropic_tensor(img, spacing, sigma, weight, align)
    cov_o, tilt_o = M.anisotropic_tensor(img, spacing, sigma, weight, align)
    assert cov.shape == img.shape + (img.ndim, img.ndim)
    assert np.max(np.abs(cov - cov_o)) <= 1e-9
    assert np.allclose(cov, np.swapaxes(cov, -1, -2), atol=1e-12)
    assert tilt_o > 0 and rel_err(tilt, tilt_o) <= 1e-10


def test_anisotropic_tensor_flat_images_give_identity():
    for img in (np.full((6, 7, 8), 0.25), np.zeros((9, 10)), np.broadcast_to(np.arange(10.0), (9, 10)).copy()):
        cov, tilt = R.anisotropic_tensor(img, None, 8.0, 400.0, 2)
        D = img.ndim
        assert np.allclose(cov, np.eye(D), atol=1e-12)
        assert tilt == DBL_LOWEST


def test_anisotropic_tensor_single_texel_axis_and_rejections():
    img = _image((1, 12, 14), 3)                       # z extent 1: the z gradient is 0
    cov, tilt = R.anisotropic_tensor(img, None, 4.0, 400.0, 2)
    cov_o, tilt_o = M.anisotropic_tensor(img, (1.0, 1.0, 1.0), 4.0, 400.0, 2)
    assert np.max(np.abs(cov - cov_o)) <= 1e-9 and tilt == tilt_o == DBL_LOWEST
    with pytest.raises(SkmError):
        R.anisotropic_tensor(img, None, -1.0, 400.0, 2)
    with pytest.raises(SkmError):
        R.anisotropic_tensor(img, None, 4.0, float("nan"), 2)


TENSOR_CASES = {
    # case 3: tensor from the smoothed target, the reference's default weights 400 / 200
    "2d_mse_target_tensor": dict(shape=(40, 44), spacing=(1.0, 1.0), config=dict(
        num_scales=2, sigma_C4=[8, 6], sigma_C0=[16, 12], cp_spacing_scaler=2.0, smoothing_variance=[1.0, 0],
        sampling_rate=[1], neighborhood_sampling=[1], num_function_evaluations=[4, 3], metric="mse",
        initial_step_size=[40000.0], tensor_weights=[400, 200])),
    "3d_ncc_target_tensor": dict(shape=(14, 16, 18), spacing=(1.0, 1.0, 1.0), config=dict(
        num_scales=2, sigma_C4=[6, 5], sigma_C0=[12, 10], cp_spacing_scaler=2.0, smoothing_variance=[1.0, 0],
        sampling_rate=[1], neighborhood_sampling=[1], num_function_evaluations=[3, 3], metric="ncc",
        reg_rd=[1e-3], initial_step_size=[1000.0], tensor_weights=[400, 200])),
}


def _pair(shape, seed=17):
    rng = np.random.default_rng(seed)
    return smooth_volume(rng, shape) * 900.0 + 100.0, smooth_volume(rng, shape) * 900.0 + 100.0


@pytest.mark.parametrize("name", sorted(TENSOR_CASES))
def test_register_with_target_tensor_matches_oracle(name):
    case = TENSOR_CASES[name]
    ref_img, tar_img = _pair(case["shape"])
    disp, rep = R.register(ref_img, tar_img, case["spacing"], None, case["config"])
    disp_o, best_o = M.register(ref_img, tar_img, case["spacing"], None, case["config"])
    assert rep["levels_done"] == case["config"]["num_scales"]
    for s, b in enumerate(best_o):
        assert rel_err(rep["best_value"][s], b) <= 1e-4, (s, rep["best_value"], best_o)
    assert np.max(np.abs(disp_o)) > 0.05
    assert max_rel(disp, disp_o) <= 1e-3


def test_register_guidance_external_tensor_and_weight_image():
    shape, spacing = (36, 40), (1.0, 1.0)
    ref_img, tar_img = _pair(shape, 5)
    rng = np.random.default_rng(8)
    guidance = smooth_volume(rng, shape)
    A = rng.normal(size=shape + (2, 2)) * 0.25
    ext = np.einsum("...ij,...kj->...ik", A, A) + 0.9 * np.eye(2)
    wimg = rng.uniform(0.6, 1.6, shape)
    base = dict(num_scales=2, sigma_C4=[8, 6], sigma_C0=[16, 12], cp_spacing_scaler=2.0, smoothing_variance=[1.0, 0],
                sampling_rate=[1], neighborhood_sampling=[1], num_function_evaluations=[3, 3], metric="mse",
                initial_step_size=[4000.0])
    runs = [
        (dict(base, tensor_weights=[300, 0]), dict(guidance_image=guidance, weight_tensor=ext)),  # case 4 then 2
        (dict(base, tensor_weights=[0]), dict(weight_tensor=ext)),                                # case 2
        (dict(base, tensor_weights=[200, 0]), dict(weight_image=wimg)),                           # weight image wins
    ]
    for cfg, kw in runs:
        disp, rep = R.register(ref_img, tar_img, spacing, None, cfg, **kw)
        disp_o, best_o = M.register(ref_img, tar_img, spacing, None, cfg, **kw)
        for s, b in enumerate(best_o):
            assert rel_err(rep["best_value"][s], b) <= 1e-4, (kw.keys(), s, rep["best_value"], best_o)
        assert np.max(np.abs(disp_o)) > 0.1
        assert max_rel(disp, disp_o) <= 1e-3
    with pytest.raises(ValueError):
        R.register(ref_img, tar_img, spacing, None, base, weight_tensor=ext[:, :-1])
