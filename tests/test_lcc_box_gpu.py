"""Box-window LCC (SKM_LCC_BOX) on the GPU against its FP64 oracle (oracle/lcc_box.py).

Every texel is a window centre with a 5^D box window; the window sums run as separable FP64 box
sums and the derivative through the generic control-point gather.  Tolerances: value 1e-5 relative,
counted centres exact, derivative 1e-4 of its largest component and 1e-4 componentwise above 1e-2
of it.  The componentwise floor is higher than the MSE / NCC tests' 1e-3: the texel coefficients of
the windows take both signs, so a control point's FP32 sum cancels more (measured on a B200:
2.2e-4 relative on 2-D components at 1e-3 of the largest, with the value equal to 1e-9).
"""
import numpy as np
import pytest

from helpers import componentwise_rel, make_problem, max_rel, rel_err
from oracle import lcc_box as LB
from skmimageregistration_b200.abi import MetricDesc, OptimizerDesc
from skmimageregistration_b200.evaluator import GpuKernelEvaluator, Optimizer, SkmError

pytestmark = pytest.mark.gpu

CASES = [
    # D, shape, sigma_c4, sigma_c0, cp_spacing, spacing
    (3, (14, 16, 18), 4.5, 9.0, 2.5, None),
    (2, (40, 44), 4.5, 9.0, 2.5, None),
    (3, (20, 22, 26), 9.0, 18.0, 4.0, (1.0, 1.0, 1.0)),     # a grid where the table path is active
]


def _check(r, g, val, count, der):
    assert r["num_pixels_counted"] == count > 0
    assert rel_err(r["measure"], val) <= 1e-5, (r["measure"], val)
    assert max_rel(g, der) <= 1e-4
    assert componentwise_rel(g, der, floor=1e-2) <= 1e-4


@pytest.mark.parametrize("D,shape,s4,s0,h,spacing", CASES)
def test_value_and_derivative_match_the_oracle(D, shape, s4, s0, h, spacing):
    pb, cp, cpw = make_problem(D, shape=shape, seed=11, sigma_c4=s4, sigma_c0=s0, cp_spacing=h, spacing=spacing)
    ev = GpuKernelEvaluator(pb)
    r, g = ev.getValueAndDerivative(GpuKernelEvaluator.LCC_BOX, cp, cpw)
    val, count, der = LB.evaluate(pb, cp, cpw)
    _check(r, g, val, count, der)
    # getValue gives the same value; a repeated call the same derivative, bit for bit
    rv = ev.getValue(GpuKernelEvaluator.LCC_BOX, cp, cpw)
    assert rv["measure"] == r["measure"] and rv["num_pixels_counted"] == r["num_pixels_counted"]
    r2, g2 = ev.getValueAndDerivative(GpuKernelEvaluator.LCC_BOX, cp, cpw)
    assert r2 == r and np.array_equal(g2, g)
    # the other metrics still run on the same evaluator afterwards
    ev.getValueAndDerivative(GpuKernelEvaluator.NCC, cp, cpw)
    ev.close()


def test_affine_intensity_change_of_the_moving_image_keeps_the_value():
    pb, cp, cpw = make_problem(3, shape=(14, 16, 18), seed=12, sigma_c4=4.5, sigma_c0=9.0, cp_spacing=2.5)
    ev = GpuKernelEvaluator(pb)
    r, _ = ev.getValueAndDerivative(GpuKernelEvaluator.LCC_BOX, cp, cpw)
    ev.close()
    pb2, _, _ = make_problem(3, shape=(14, 16, 18), seed=12, sigma_c4=4.5, sigma_c0=9.0, cp_spacing=2.5,
                             coeffs=3.0 * pb.moving_coefficients + 5.0)
    ev2 = GpuKernelEvaluator(pb2)
    r2, _ = ev2.getValueAndDerivative(GpuKernelEvaluator.LCC_BOX, cp, cpw)
    ev2.close()
    assert r2["num_pixels_counted"] == r["num_pixels_counted"]
    assert rel_err(r2["measure"], r["measure"]) <= 1e-5


def test_subsampled_evaluator_is_rejected():
    pb, cp, cpw = make_problem(3, shape=(14, 16, 18), subsample=2, seed=13)
    ev = GpuKernelEvaluator(pb)
    with pytest.raises(SkmError) as ei:
        ev.getValueAndDerivative(GpuKernelEvaluator.LCC_BOX, cp, cpw)
    assert ei.value.code == 1
    ev.close()


def test_device_optimizer_lowers_the_box_lcc():
    pb, _, cpw = make_problem(3, shape=(14, 16, 18), seed=14, sigma_c4=4.5, sigma_c0=9.0, cp_spacing=2.5,
                              weights=False)
    P = pb.num_parameters
    m = MetricDesc.make("lcc_box", rd=1e-3)
    o = OptimizerDesc.make(a=5.0, number_of_iterations=30)
    ev = GpuKernelEvaluator(pb)
    opt = Optimizer(ev, o, m, np.zeros(P), cpw)
    opt.run(30)
    best = opt.parameters(best=True)
    v0, _, _ = LB.evaluate(pb, np.zeros((pb.C, pb.D)), cpw, derivative=False)
    v1, _, _ = LB.evaluate(pb, best.reshape(pb.D, pb.C).T.copy(), cpw, derivative=False)
    assert v1 < v0
    opt.close()
    ev.close()
