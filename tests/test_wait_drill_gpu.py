"""The bounded-wait error path of the tensor-core kernels, exercised without any GPU fault.

Every mbarrier wait in the tcgen05 kernels gives up after a bounded time; the kernel then waits
(bounded) for its own copies and MMAs in flight, frees its tensor memory and returns, and the
call reports SKM_ERR_TIMEOUT with its results discarded.  skm_evaluator_wait_drill makes exactly
one wait run out on purpose: in the contrib GEMM, block 0's first producer group withholds a
shared-memory stage on which no copy and no MMA depends (a flag nothing sets), with a 5 ms wait
limit for that launch.  The test checks the status, that nothing of the failed call is returned,
and that the next call on the same evaluator is correct (bitwise equal to a fresh evaluator, and
within the parity tolerances of the FP64 oracle).
"""
import numpy as np
import pytest

from helpers import make_problem, max_rel, rel_err
from oracle import oracle as O
from skmimageregistration_b200 import abi
from skmimageregistration_b200.evaluator import GpuKernelEvaluator, SkmError

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("metric", [abi.MSE, abi.NCC])
def test_wait_that_runs_out_reports_timeout_and_evaluator_recovers(metric):
    pb, cp, cpw = make_problem(3, shape=(20, 22, 26), seed=61, sigma_c4=9.0, sigma_c0=18.0, cp_spacing=4.0,
                               spacing=(1.0, 1.0, 1.0))
    ev = GpuKernelEvaluator(pb)
    assert ev.path() == GpuKernelEvaluator.TABLE_TC
    ev.SetRegularizerRD(1e-2)
    sentinel = np.full(pb.num_parameters, 1234.5)
    ev.wait_drill(True)
    with pytest.raises(SkmError) as exc:
        ev.getValueAndDerivative(metric, cp, cpw, derivatives=sentinel)
    assert exc.value.code == abi.SKM_ERR_TIMEOUT
    assert np.all(sentinel == 1234.5)                  # the failed call's derivative is discarded
    # the drill disarmed itself; the same evaluator computes the right result next
    r, g = ev.getValueAndDerivative(metric, cp, cpw)
    fresh = GpuKernelEvaluator(pb)
    fresh.SetRegularizerRD(1e-2)
    rf, gf = fresh.getValueAndDerivative(metric, cp, cpw)
    assert r == rf
    assert np.array_equal(g, gf)
    orc = O.Oracle(pb)
    orc.set_regularizers(rd=1e-2)
    ro, go = orc.evaluate(metric, cp, cpw)
    assert r["num_pixels_counted"] == ro["num_pixels_counted"]
    assert rel_err(r["measure"], ro["measure"]) <= 1e-5
    assert max_rel(g, go) <= 1e-4


def test_wait_drill_needs_the_tensor_core_path():
    pb, cp, cpw = make_problem(3, seed=62)
    ev = GpuKernelEvaluator(pb)
    assert ev.path() == GpuKernelEvaluator.GENERIC
    with pytest.raises(SkmError) as exc:
        ev.wait_drill(True)
    assert exc.value.code == abi.SKM_ERR_UNSUPPORTED
