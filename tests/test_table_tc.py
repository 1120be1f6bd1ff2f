"""Tensor-core GEMMs of the phase-table path at the benchmark sizes.

At these sizes every CTA of the persistent tensor-core kernels works through several tiles,
so both TMEM accumulators, every shared-memory stage and both mbarrier parities are in use
(the small parity cases run one tile per CTA).  The tensor-core path (3xTF32 products, FP32
accumulation) is compared with the CUDA-core table path (FP32 FMA) on the same inputs:
  * metric value: relative difference <= 1e-5, pixel counts exact
  * derivative:   max |g_tc - g_cc| <= 1e-4 * max |g_cc|
and both against the generic kernels with the same bounds.
"""
import numpy as np
import pytest

from helpers import max_rel, rel_err
from skmimageregistration_b200 import workloads
from skmimageregistration_b200.evaluator import GpuKernelEvaluator

pytestmark = pytest.mark.gpu


def _params(pb, seed, scale):
    rng = np.random.default_rng(seed)
    cp = rng.normal(0.0, scale, (pb.C, pb.D))
    cpw = rng.uniform(0.5, 1.5, pb.C)
    return np.ascontiguousarray(cp), np.ascontiguousarray(cpw)


@pytest.mark.parametrize("name", ["ncc128", "mse2d"])
def test_tensor_core_table_matches_cuda_core_table_at_bench_size(name):
    pb, m, _, _ = workloads.make(name, seed=0)
    ev = GpuKernelEvaluator(pb)
    if name == "ncc128":
        ev.SetRegularizerRD(1e-3)
    metric = m.metric
    for seed, scale in ((1, 0.5), (2, 2.0)):
        cp, cpw = _params(pb, seed, scale)
        assert ev.path(GpuKernelEvaluator.AUTO) == GpuKernelEvaluator.TABLE_TC
        r_tc, g_tc = ev.getValueAndDerivative(metric, cp, cpw)
        assert ev.path(GpuKernelEvaluator.REQ_TABLE_CUDA_CORES) == GpuKernelEvaluator.TABLE
        r_cc, g_cc = ev.getValueAndDerivative(metric, cp, cpw)
        assert ev.path(GpuKernelEvaluator.REQ_GENERIC) == GpuKernelEvaluator.GENERIC
        r_g, g_g = ev.getValueAndDerivative(metric, cp, cpw)
        assert r_tc["num_pixels_counted"] == r_cc["num_pixels_counted"] == r_g["num_pixels_counted"]
        assert rel_err(r_tc["measure"], r_cc["measure"]) <= 1e-5
        assert rel_err(r_tc["measure"], r_g["measure"]) <= 1e-5
        assert max_rel(g_tc, g_cc) <= 1e-4
        assert max_rel(g_tc, g_g) <= 1e-4
        assert np.all(np.isfinite(g_tc))


def test_tensor_core_table_value_only_matches_derivative_call():
    pb, m, _, _ = workloads.make("ncc128", seed=0)
    ev = GpuKernelEvaluator(pb)
    ev.SetRegularizerRD(1e-3)
    cp, cpw = _params(pb, 4, 1.0)
    assert ev.path() == GpuKernelEvaluator.TABLE_TC
    r1 = ev.getValue(m.metric, cp, cpw)
    r2, _ = ev.getValueAndDerivative(m.metric, cp, cpw)
    assert r1["num_pixels_counted"] == r2["num_pixels_counted"]
    assert r1["measure"] == r2["measure"]
    assert r1["reg_value_rd"] == r2["reg_value_rd"]


# the table path takes spacing ratios 1, 2, 4, 8 per axis, so phase counts below 8 occur for
# h = 1 (one phase) and, in 2-D, h = 2 (four phases)
@pytest.mark.parametrize("D,h,shape", [(2, 1, (30, 34)), (2, 2, (40, 46)), (3, 1, (12, 14, 16)), (3, 2, (18, 20, 22))])
def test_tensor_core_variants_for_small_phase_counts(D, h, shape):
    """Phase counts that are not multiples of 8 (or of 4) keep the direct record loads (and the
    direct stores of u) of the tensor-core kernels; the others use the record ring and the staged
    stores.  Either way the results match the CUDA-core table path and the generic kernels."""
    from helpers import make_problem
    pb, cp, cpw = make_problem(D, "stationary", shape=shape, seed=11 + h, sigma_c4=3.0 * h, sigma_c0=6.0 * h,
                               cp_spacing=float(h), spacing=(1.0,) * D, origin=tuple([0.5, -1.0, 2.0][:D]))
    ev = GpuKernelEvaluator(pb)
    assert ev.path(GpuKernelEvaluator.AUTO) == GpuKernelEvaluator.TABLE_TC
    info = ev.describe()
    nph = h ** D
    assert info["table_phases"] == nph
    assert info["tc_record_slots"] == 0 if nph % 8 else info["tc_record_slots"] >= 2
    assert info["tc_u_staging"] == 0 if nph % 4 else info["tc_u_staging"] >= 1
    assert info["tc_region_buffers"] in (2, 3)
    for metric in (GpuKernelEvaluator.MSE, GpuKernelEvaluator.NCC):
        r_tc, g_tc = ev.getValueAndDerivative(metric, cp, cpw)
        assert ev.path(GpuKernelEvaluator.REQ_TABLE_CUDA_CORES) == GpuKernelEvaluator.TABLE
        r_cc, g_cc = ev.getValueAndDerivative(metric, cp, cpw)
        assert ev.path(GpuKernelEvaluator.REQ_GENERIC) == GpuKernelEvaluator.GENERIC
        r_g, g_g = ev.getValueAndDerivative(metric, cp, cpw)
        ev.path(GpuKernelEvaluator.AUTO)
        assert r_tc["num_pixels_counted"] == r_cc["num_pixels_counted"] == r_g["num_pixels_counted"] > 0
        assert rel_err(r_tc["measure"], r_cc["measure"]) <= 1e-5
        assert rel_err(r_tc["measure"], r_g["measure"]) <= 1e-5
        assert max_rel(g_tc, g_cc) <= 1e-4
        assert max_rel(g_tc, g_g) <= 1e-4


def test_brick_partials_match_tap_gather_and_oracle_at_bench_size():
    """The contrib GEMM's brick partials (scattered per brick into its control-point patch, summed
    by the gather; path request 3) against the per-tap Contrib array with the tap gather (the
    automatic path) and against the FP64 oracle, at ncc128 with RD; repeat calls bitwise identical
    (no atomics)."""
    from oracle import oracle as O
    pb, m, _, _ = workloads.make("ncc128", seed=0)
    ev = GpuKernelEvaluator(pb)
    ev.SetRegularizerRD(1e-3)
    orc = O.Oracle(pb)
    orc.set_regularizers(rd=1e-3)
    cp, cpw = _params(pb, 5, 1.0)
    assert ev.path(GpuKernelEvaluator.AUTO) == GpuKernelEvaluator.TABLE_TC
    assert ev.describe()["tc_contrib_bricks"] == 0
    r_t, g_t = ev.getValueAndDerivative(m.metric, cp, cpw)
    assert ev.path(GpuKernelEvaluator.REQ_TABLE_TC_BRICKS) == GpuKernelEvaluator.TABLE_TC
    assert ev.describe()["tc_contrib_bricks"] == 1
    r_b, g_b = ev.getValueAndDerivative(m.metric, cp, cpw)
    r_b2, g_b2 = ev.getValueAndDerivative(m.metric, cp, cpw)
    assert np.array_equal(g_b, g_b2) and r_b["measure"] == r_b2["measure"]
    ro, go = orc.evaluate(m.metric, cp, cpw)
    assert r_b["measure"] == r_t["measure"]                 # the value pass is the same
    assert r_b["num_pixels_counted"] == r_t["num_pixels_counted"] == ro["num_pixels_counted"]
    assert rel_err(r_b["reg_value_rd"], ro["reg_value_rd"]) <= 1e-5
    assert max_rel(g_b, g_t) <= 1e-5
    assert max_rel(g_b, go) <= 1e-4
    assert max_rel(g_t, go) <= 1e-4
