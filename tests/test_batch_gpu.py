"""Batched registration: many pairs of uneven sizes in one persistent kernel per iteration.

Each pair's value and derivative inside the batch are compared with the FP64 oracle
(metric level: measure + regularizers, negated gradient) and with a single-pair evaluation on the
CUDA-core table path; a few optimizer iterations of the batch are compared with the single-pair
device optimizer and the FP64 oracle optimizer.  Tolerances as in the parity tests: values 1e-5
relative, derivatives 1e-4 of the largest component (and componentwise above 1e-2 of it).
"""
import numpy as np
import pytest

from helpers import componentwise_rel, make_problem, max_rel, rel_err
from oracle import oracle as O
from skmimageregistration_b200.abi import MetricDesc, OptimizerDesc
from skmimageregistration_b200.evaluator import Batch, GpuKernelEvaluator, Optimizer

pytestmark = pytest.mark.gpu

SHAPES = [(20, 24, 28), (24, 20, 33), (29, 27, 21), (17, 25, 24), (32, 21, 26), (22, 31, 30)]


def _pairs(seed=0):
    problems, metrics, params, cpws = [], [], [], []
    for i, shape in enumerate(SHAPES):
        pb, cp, cpw = make_problem(3, shape=shape, seed=seed + 200 + i, sigma_c4=9.0, sigma_c0=18.0, cp_spacing=4.0,
                                   spacing=(1.0, 1.0, 1.0), origin=(0.5 * i, -1.0, 2.0))
        problems.append(pb)
        if i % 2 == 0:
            metrics.append(MetricDesc.make("ncc", rd=1e-2, l1=1e-4))
        else:
            metrics.append(MetricDesc.make("mse", rkhs=1e-2, l2=1e-4, pg=1e-3, pg_scaling=0.5))
        params.append(np.ascontiguousarray(cp.T.reshape(-1) * 0.5))
        cpws.append(cpw)
    return problems, metrics, params, cpws


def test_batch_evaluation_matches_oracle_and_single_pair():
    problems, metrics, params, cpws = _pairs()
    opt = OptimizerDesc.make(a=50.0, number_of_iterations=1000)
    b = Batch(problems, metrics, opt, initial=params, cpws=cpws)
    info = b.describe()
    assert info["pairs"] == len(SHAPES) and info["candidates"] >= 2
    b.evaluate()
    for i, pb in enumerate(problems):
        v, g = b.result(i)
        orc = O.Oracle(pb)
        vo, go = orc.metric(metrics[i], params[i], cpws[i])
        orc.close()
        assert v["num_pixels_counted"] == vo["num_pixels_counted"]
        for k in ("value", "measure", "reg_value"):
            assert rel_err(v[k], vo[k]) <= 1e-5, (i, k, v[k], vo[k])
        assert max_rel(g, go) <= 1e-4, i
        assert componentwise_rel(g, go, 1e-2) <= 1e-4, i
        ev = GpuKernelEvaluator(pb)
        assert ev.path(GpuKernelEvaluator.REQ_TABLE_CUDA_CORES) == GpuKernelEvaluator.TABLE
        vs, gs = ev.metric(metrics[i], params[i], cpws[i])
        assert v["num_pixels_counted"] == vs["num_pixels_counted"]
        assert rel_err(v["value"], vs["value"]) <= 1e-6
        assert max_rel(g, gs) <= 1e-5
    # deterministic: a second evaluation gives the same bits
    first = [b.result(i) for i in range(len(problems))]
    b.evaluate()
    for i in range(len(problems)):
        v, g = b.result(i)
        assert v == first[i][0] and np.array_equal(g, first[i][1])


def test_batch_optimizer_iterations_match_single_pair_and_oracle():
    problems, metrics, params, cpws = _pairs(seed=7)
    opt = OptimizerDesc.make(a=20.0, number_of_iterations=1000)
    b = Batch(problems, metrics, opt, initial=params, cpws=cpws)
    iters = 4
    b.run(iters)
    for i, pb in enumerate(problems):
        ev = GpuKernelEvaluator(pb)
        ev.path(GpuKernelEvaluator.REQ_TABLE_CUDA_CORES)
        o = Optimizer(ev, opt, metrics[i], params[i], cpws[i])
        o.run(iters)
        s_b, s_o = b.state(i), o.state()
        assert s_b["iteration"] == s_o["iteration"] == iters
        assert rel_err(s_b["value"], s_o["value"]) <= 1e-5
        assert rel_err(s_b["best_value"], s_o["best_value"]) <= 1e-5
        assert max_rel(b.parameters(i), o.parameters()) <= 1e-4
        assert max_rel(b.parameters(i, best=True), o.parameters(best=True)) <= 1e-4
        orc = O.Oracle(pb)
        oo = O.OracleOptimizer(orc, opt, metrics[i], params[i], cpws[i])
        oo.run(iters)
        assert max_rel(b.parameters(i), oo.position) <= 1e-4
        orc.close()
        o.close()
        ev.close()


def test_batch_rejects_pairs_off_the_table_path():
    pb, cp, cpw = make_problem(3, seed=3)                 # control spacing 2 x 1.1 x 0.9 voxels: no table
    with pytest.raises(Exception) as exc:
        Batch([pb], MetricDesc.make("ncc"), OptimizerDesc.make())
    assert "phase-table" in str(exc.value)
