"""Multi-scale driver and its preprocessing on the GPU against the FP64 restatements.

Tolerances:
  * smoothing, threshold + rescale (FP64 on both sides): max |a - b| <= 1e-10 * max |b|
  * registration: displacement max |u - u_ref| <= 1e-3 * max |u_ref| and per-level best value
    relative error <= 1e-4 after a few optimizer iterations per level (the FP32 evaluator and the
    FP64 oracle drift apart through the adaptive step sizes, as in the optimizer parity tests).
"""
import numpy as np
import pytest

from helpers import max_rel, rel_err, smooth_volume
from oracle import multiscale as M
from skmimageregistration_b200 import register as R
from skmimageregistration_b200.evaluator import SkmError

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape,spacing", [((40, 44), (1.0, 1.5)), ((14, 16, 18), (1.0, 0.8, 1.2))])
@pytest.mark.parametrize("variance", [0.3, 2.0, 9.0])
def test_gaussian_smooth_matches_oracle(shape, spacing, variance):
    rng = np.random.default_rng(3)
    img = rng.normal(0, 1, shape) + smooth_volume(rng, shape)
    got = R.gaussian_smooth(img, spacing, variance)
    ref = M.gaussian_smooth(img, spacing, variance)
    assert max_rel(got, ref) <= 1e-10


def test_threshold_rescale_matches_oracle():
    rng = np.random.default_rng(5)
    img = rng.normal(500, 1500, (20, 24, 28))
    for th in ((-1500, 3500), None):
        got = R.threshold_rescale(img, th)
        ref = M.threshold_rescale(img, th)
        assert max_rel(got, ref) <= 1e-10
    with pytest.raises(SkmError):
        R.threshold_rescale(np.full((8, 8), 5000.0), (-1500, 3500))


CASES = {
    # generic kernels: subsampled NCC with RD, smoothing on the first level
    "2d_ncc_generic": dict(shape=(40, 44), spacing=(1.0, 1.0), config=dict(
        num_scales=2, sigma_C4=[8, 6], sigma_C0=[16, 12], cp_spacing_scaler=2.0, smoothing_variance=[1.0, 0],
        sampling_rate=[2, 1], neighborhood_sampling=[1], num_function_evaluations=[4, 3], metric="ncc",
        reg_rd=[1e-3], initial_step_size=[1000.0], tensor_weights=[0])),
    # phase-table path with the tensor-core GEMMs (control spacing 2 voxels, every voxel sampled)
    "3d_mse_table": dict(shape=(20, 22, 26), spacing=(1.0, 1.0, 1.0), config=dict(
        num_scales=2, sigma_C4=[8, 8], sigma_C0=[16, 16], cp_spacing_scaler=4.0, smoothing_variance=[2.0, 0],
        sampling_rate=[1], neighborhood_sampling=[1], num_function_evaluations=[3, 3], metric="mse",
        initial_step_size=[400.0], tensor_weights=[0])),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_register_matches_oracle_driver(name):
    case = CASES[name]
    rng = np.random.default_rng(17)
    ref_img = smooth_volume(rng, case["shape"]) * 900.0 + 100.0
    tar_img = smooth_volume(rng, case["shape"]) * 900.0 + 100.0
    disp, rep = R.register(ref_img, tar_img, case["spacing"], None, case["config"])
    disp_o, best_o = M.register(ref_img, tar_img, case["spacing"], None, case["config"])
    assert rep["levels_done"] == case["config"]["num_scales"]
    assert rep["iterations"] == list(case["config"]["num_function_evaluations"])
    for s, b in enumerate(best_o):
        assert rel_err(rep["best_value"][s], b) <= 1e-4, (s, rep["best_value"], best_o)
    assert np.max(np.abs(disp_o)) > 0.2                   # the registration moved by a fraction of a voxel
    assert max_rel(disp, disp_o) <= 1e-3
