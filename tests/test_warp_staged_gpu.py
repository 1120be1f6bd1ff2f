"""The warp kernel that stages the moving image's coefficient boxes by TMA (3-D tensor-core path).

It must give the same metric and derivative as the CUDA-core table path (global-memory B-spline
rows) whatever the displacement: inside the staged box's margin, beyond it (those stencils read
global memory), with a previous-level displacement field, and when the moving image's grid is
not the fixed image's (spacing ratio and origin shift change the box origins).  Tolerances as the
tensor-core table tests: value 1e-5 relative, derivative 1e-4 of its maximum, pixel counts exact.
"""
import numpy as np
import pytest

from helpers import max_rel, rel_err, smooth_volume
from skmimageregistration_b200 import workloads
from skmimageregistration_b200.evaluator import GpuKernelEvaluator, bspline_coefficients
from skmimageregistration_b200.problem import Problem

pytestmark = pytest.mark.gpu


def _compare(ev, metric, cp, cpw, df=None, df_geometry=None):
    assert ev.path(GpuKernelEvaluator.AUTO) == GpuKernelEvaluator.TABLE_TC
    assert ev.describe()["warp_staged"] == 1
    r_tc, g_tc = ev.getValueAndDerivative(metric, cp, cpw, df, df_geometry)
    assert ev.path(GpuKernelEvaluator.REQ_TABLE_CUDA_CORES) == GpuKernelEvaluator.TABLE
    r_cc, g_cc = ev.getValueAndDerivative(metric, cp, cpw, df, df_geometry)
    ev.path(GpuKernelEvaluator.AUTO)
    assert r_tc["num_pixels_counted"] == r_cc["num_pixels_counted"] > 0
    assert rel_err(r_tc["measure"], r_cc["measure"]) <= 1e-5
    assert max_rel(g_tc, g_cc) <= 1e-4
    return r_tc


@pytest.mark.parametrize("scale", [0.2, 3.0, 12.0])
def test_staged_warp_matches_global_rows_for_small_and_large_displacements(scale):
    pb, m, _, _ = workloads.make("ncc128", seed=0)
    ev = GpuKernelEvaluator(pb)
    rng = np.random.default_rng(7)
    cp = np.ascontiguousarray(rng.normal(0.0, scale, (pb.C, pb.D)))
    cpw = np.ones(pb.C)
    u = ev.evaluateDisplacementField(cp, cpw)
    if scale > 10:
        assert np.max(np.abs(u)) > 8.0                     # far beyond the 3-voxel margin of the box
    _compare(ev, m.metric, cp, cpw)
    ev.close()


def test_staged_warp_with_a_displacement_field_and_another_moving_grid():
    rng = np.random.default_rng(3)
    shape = (40, 48, 56)
    fixed = smooth_volume(rng, shape)
    moving = smooth_volume(rng, shape)
    # moving grid: 0.8 mm voxels shifted by (1.3, -2.1, 0.7) mm; fixed grid 1 mm; control spacing 4 mm
    pb = Problem(fixed=fixed, moving_coefficients=bspline_coefficients(moving), spacing=(1.0, 1.0, 1.0),
                 origin=(0.0, 0.0, 0.0), sigma_c0=24.0, sigma_c4=12.0, cp_spacing=4.0,
                 moving_origin=(1.3, -2.1, 0.7), moving_spacing=(0.8, 0.8, 0.8))
    ev = GpuKernelEvaluator(pb)
    cp = np.ascontiguousarray(rng.normal(0.0, 1.5, (pb.C, pb.D)))
    cpw = rng.uniform(0.5, 1.5, pb.C)
    df = np.ascontiguousarray(rng.normal(0.0, 2.0, shape + (3,)))
    for metric in (GpuKernelEvaluator.MSE, GpuKernelEvaluator.NCC):
        _compare(ev, metric, cp, cpw)
        _compare(ev, metric, cp, cpw, df, pb.fixed_geometry())
    ev.close()
