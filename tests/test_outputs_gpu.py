"""Output images and checkpoint/restart of the registration driver on the GPU.

Tolerances: warped image and Jacobian determinant (FP64 on both sides): max |a - b| <= 1e-12 of
max |b|; a restarted run reproduces the full run's field to 1e-12 of its maximum (same inputs,
same kernels, so in practice bit for bit)."""
import numpy as np
import pytest

from helpers import max_rel, smooth_volume
from oracle import multiscale as M
from skmimageregistration_b200 import register as R
from skmimageregistration_b200.evaluator import SkmError

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("order", [1, 3])
@pytest.mark.parametrize("D", [2, 3])
def test_warp_image_matches_oracle(order, D):
    rng = np.random.default_rng(20 + D)
    ishape = (30, 34) if D == 2 else (12, 14, 16)
    fshape = (26, 31) if D == 2 else (11, 15, 13)
    img = smooth_volume(rng, ishape) + 0.1 * rng.normal(size=ishape)
    u = rng.normal(size=fshape + (D,)) * 2.5                 # pushes some positions outside the image
    isp, iog = (1.0, 1.2, 0.9)[:D], (0.5, -1.0, 2.0)[:D]
    fsp, fog = (1.1, 1.0, 1.05)[:D], (1.0, 0.0, 1.5)[:D]
    got = R.warp_image(img, u, isp, iog, fsp, fog, order=order, default_value=-3.0)
    ref = M.warp_image(img, u, isp, iog, fsp, fog, order=order, default_value=-3.0)
    assert np.any(ref == -3.0) and np.any(ref != -3.0)
    assert max_rel(got, ref) <= 1e-12


def test_warp_image_rejections():
    img = np.zeros((1, 8))
    with pytest.raises(SkmError):
        R.warp_image(img, np.zeros((1, 8, 2)), order=3)          # cubic needs 2 texels per axis
    with pytest.raises(SkmError):
        R.warp_image(np.zeros((8, 8)), np.zeros((8, 8, 2)), order=2)
    out = R.warp_image(img, np.zeros((1, 8, 2)), order=1)
    assert np.array_equal(out, img)


@pytest.mark.parametrize("D", [2, 3])
def test_jacobian_determinant_matches_oracle(D):
    rng = np.random.default_rng(30 + D)
    shape = (33, 29) if D == 2 else (9, 12, 11)
    u = rng.normal(size=shape + (D,)) * 0.4
    sp = (0.8, 1.3, 2.0)[:D]
    got = R.jacobian_determinant(u, sp)
    ref = M.jacobian_determinant(u, sp)
    assert max_rel(got, ref) <= 1e-12


def test_restart_reproduces_the_full_run_and_levels_are_reported():
    rng = np.random.default_rng(17)
    ref = smooth_volume(rng, (14, 16, 18)) * 900 + 100
    tar = smooth_volume(rng, (14, 16, 18)) * 900 + 100
    cfg = dict(num_scales=3, sigma_C4=[8, 6, 5], sigma_C0=[16, 12, 10], cp_spacing_scaler=2.0,
               smoothing_variance=[1.0, 0.5, 0], sampling_rate=[1], neighborhood_sampling=[1],
               num_function_evaluations=[3, 3, 2], metric="ncc", reg_rd=[1e-3], initial_step_size=[1000.0],
               tensor_weights=[400, 200, 100])
    levels = {}
    full, rep = R.register(ref, tar, (1.0, 1.0, 1.0), None, cfg, on_level=lambda s, f: levels.__setitem__(s, f))
    assert sorted(levels) == [0, 1, 2] and rep["first_level"] == 0
    assert np.array_equal(levels[2], full)
    again, rep2 = R.register(ref, tar, (1.0, 1.0, 1.0), None, dict(cfg, restart_at=3),
                             initial_displacement=levels[1])
    assert rep2["first_level"] == 2 and rep2["levels_done"] == 3 and rep2["iterations"][:2] == [0, 0]
    assert max_rel(again, full) <= 1e-12
    # restart_at without a field starts from the first level, as SKMReg does when the file is missing
    fresh, rep3 = R.register(ref, tar, (1.0, 1.0, 1.0), None, dict(cfg, restart_at=2))
    assert rep3["first_level"] == 0 and max_rel(fresh, full) <= 1e-12
