"""The CUDA path against the reference's own GpuKernelEvaluator on the same inputs.

The reference evaluator (include/cuda/GpuEvaluator.cu, unmodified, double build with the
reference's -use_fast_math, compiled for sm_100a into oracle/_ref by oracle/Makefile) runs on
the same GPU.  Same tolerances as against the FP64 oracle: values 1e-5 relative, derivatives
1e-4 of the largest component, transform 1e-5, pixel counts exact.  Subsampled cases check
that both draw the same PCG32 sample shifts (the driver refuses draws that would make the
reference read out of bounds).
"""
import os

import numpy as np
import pytest

from helpers import make_problem, max_rel, rel_err
from oracle import oracle as O
from skmimageregistration_b200 import abi
from skmimageregistration_b200.evaluator import GpuKernelEvaluator

pytestmark = pytest.mark.gpu


def _ref(pb):
    if not os.path.exists(O.ref_gpu_path(pb.D, True)):
        pytest.skip("reference evaluator not built (oracle/_ref)")
    return O.RefGpu(pb, double=True)


@pytest.mark.parametrize("D", [2, 3])
@pytest.mark.parametrize("kind", ["stationary", "weight_image", "weight_tensor"])
@pytest.mark.parametrize("metric", [abi.MSE, abi.NCC])
@pytest.mark.parametrize("sub", [1, 2])
def test_matches_reference_evaluator(D, kind, metric, sub):
    shape = (14, 16, 18) if D == 3 else (40, 44)
    pb, cp, cpw = make_problem(D, kind, subsample=sub, shape=shape, seed=101)
    ref = _ref(pb)
    ev = GpuKernelEvaluator(pb)
    ev.SetRegularizerRD(0.05)
    ref.set_regularizers(rd=0.05)
    for call in range(2):
        r, g = ev.getValueAndDerivative(metric, cp, cpw)
        rr, gr = ref.evaluate(metric, cp, cpw)
        assert r["num_pixels_counted"] == rr["num_pixels_counted"]
        assert rel_err(r["measure"], rr["measure"]) <= 1e-5, (r, rr)
        assert rel_err(r["reg_value_rd"], rr["reg_value_rd"]) <= 1e-5
        assert max_rel(g, gr) <= 1e-4


@pytest.mark.parametrize("D", [2, 3])
@pytest.mark.parametrize("request_, expected", [(GpuKernelEvaluator.AUTO, GpuKernelEvaluator.TABLE_TC),
                                                (GpuKernelEvaluator.REQ_TABLE_CUDA_CORES, GpuKernelEvaluator.TABLE)])
def test_table_path_matches_reference_evaluator(D, request_, expected):
    shape = (20, 22, 26) if D == 3 else (40, 44)
    pb, cp, cpw = make_problem(D, "stationary", shape=shape, seed=103, sigma_c4=9.0, sigma_c0=18.0, cp_spacing=4.0,
                               spacing=(1.0,) * D)
    ref = _ref(pb)
    ev = GpuKernelEvaluator(pb)
    assert ev.path(request_) == expected
    ev.SetRegularizerRD(0.05)
    ref.set_regularizers(rd=0.05)
    for metric in (abi.MSE, abi.NCC):
        r, g = ev.getValueAndDerivative(metric, cp, cpw)
        rr, gr = ref.evaluate(metric, cp, cpw)
        assert r["num_pixels_counted"] == rr["num_pixels_counted"]
        assert rel_err(r["measure"], rr["measure"]) <= 1e-5
        assert max_rel(g, gr) <= 1e-4


@pytest.mark.parametrize("D", [2, 3])
def test_lcc_matches_reference_evaluator(D):
    shape = (10, 11, 12) if D == 3 else (24, 26)
    pb, cp, cpw = make_problem(D, "stationary", subsample=2, nbh=2, shape=shape, seed=105, sigma_c4=3.0,
                               sigma_c0=6.0, cp_spacing=1.5)
    ref = _ref(pb)
    ev = GpuKernelEvaluator(pb)
    r, g = ev.getValueAndDerivative(abi.LCC, cp, cpw)
    rr, gr = ref.evaluate(abi.LCC, cp, cpw)
    assert r["num_pixels_counted"] == rr["num_pixels_counted"]
    assert rel_err(r["measure"], rr["measure"]) <= 1e-5
    assert max_rel(g, gr) <= 1e-4


@pytest.mark.parametrize("D", [2, 3])
def test_displacement_field_matches_reference_evaluator(D):
    pb, cp, cpw = make_problem(D, "stationary", seed=107)
    ref = _ref(pb)
    ev = GpuKernelEvaluator(pb)
    rng = np.random.default_rng(1)
    df = rng.normal(0, 0.5, (pb.n_texels, D))
    assert max_rel(ev.evaluateDisplacementField(cp, cpw, df), ref.displacement_field(cp, cpw, df)) <= 1e-5


@pytest.mark.parametrize("D,shape,cp_spacing", [(2, (48, 52), 1.5), (3, (24, 24, 24), 2.0)])
@pytest.mark.parametrize("kind", ["weight_tensor", "weight_image"])
def test_lcc_nonstationary_matches_reference_evaluator(D, shape, cp_spacing, kind):
    """LCC over the anisotropic and the weight-image kernels (config 3's combination is the
    anisotropic one) at 24^3, subsample 2, neighbourhood stride 2, random control-point weights."""
    pb, cp, cpw = make_problem(D, kind, subsample=2, nbh=2, shape=shape, seed=109, sigma_c4=3.0, sigma_c0=6.0,
                               cp_spacing=cp_spacing)
    ref = _ref(pb)
    ev = GpuKernelEvaluator(pb)
    for call in range(2):
        r, g = ev.getValueAndDerivative(abi.LCC, cp, cpw)
        rr, gr = ref.evaluate(abi.LCC, cp, cpw)
        assert r["num_pixels_counted"] == rr["num_pixels_counted"]
        assert rel_err(r["measure"], rr["measure"]) <= 1e-5
        assert max_rel(g, gr) <= 1e-4
