"""CUDA evaluation path (through the C-ABI) against the FP64 oracle.

Tolerances (stated against the FP64 oracle, FP32 arithmetic on the device):
  * transform / displacement field: max |u - u_ref| <= 1e-5 * max |u_ref|
  * metric values and regularizer values: relative error <= 1e-5
  * derivatives: max |g - g_ref| <= 1e-4 * max |g_ref|
  * pixel counts: exact
"""
import numpy as np
import pytest

from helpers import make_problem, max_rel, rel_err
from oracle import oracle as O
from skmimageregistration_b200 import abi
from skmimageregistration_b200.abi import MetricDesc, OptimizerDesc
from skmimageregistration_b200.evaluator import GpuKernelEvaluator, Optimizer, bspline_coefficients

pytestmark = pytest.mark.gpu

TOL_FIELD = 1e-5
TOL_VALUE = 1e-5
TOL_DERIV = 1e-4

KINDS = ["stationary", "weight_image", "weight_tensor"]


def _df_for(pb, seed=3):
    rng = np.random.default_rng(seed)
    return rng.normal(0, 0.7, (pb.n_texels, pb.D))


@pytest.mark.parametrize("D", [2, 3])
@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("with_df", [False, True])
def test_displacement_field(D, kind, with_df):
    pb, cp, cpw = make_problem(D, kind, seed=11)
    df = _df_for(pb) if with_df else None
    ev = GpuKernelEvaluator(pb)
    got = ev.evaluateDisplacementField(cp, cpw, df)
    ref = O.Oracle(pb).displacement_field(cp, cpw, df)
    assert max_rel(got, ref) <= TOL_FIELD


@pytest.mark.parametrize("D", [2, 3])
@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("metric", [abi.MSE, abi.NCC])
@pytest.mark.parametrize("sub", [1, 3])
def test_value_and_derivative(D, kind, metric, sub):
    pb, cp, cpw = make_problem(D, kind, subsample=sub, seed=5 + sub)
    ev = GpuKernelEvaluator(pb)
    orc = O.Oracle(pb)
    df = _df_for(pb, 7)
    for call in range(2):            # second call redraws the sample shifts
        r, g = ev.getValueAndDerivative(metric, cp, cpw, df)
        ro, go = orc.evaluate(metric, cp, cpw, df)
        assert r["num_pixels_counted"] == ro["num_pixels_counted"]
        assert rel_err(r["measure"], ro["measure"]) <= TOL_VALUE, (r, ro)
        assert max_rel(g, go) <= TOL_DERIV


@pytest.mark.parametrize("D", [2, 3])
@pytest.mark.parametrize("metric", [abi.MSE, abi.NCC])
def test_get_value_matches_value_and_derivative(D, metric):
    """GetValue == GetValueAndDerivative value (itkFiniteDifferenceTest.cpp:188-217)."""
    pb, cp, cpw = make_problem(D, seed=21)
    ev = GpuKernelEvaluator(pb)
    ev.SetRegularizerRD(1e-2)
    v = ev.getValue(metric, cp, cpw)
    r, _ = ev.getValueAndDerivative(metric, cp, cpw)
    assert v["measure"] == r["measure"]
    assert v["reg_value_rd"] == pytest.approx(r["reg_value_rd"], rel=1e-12)


@pytest.mark.parametrize("D", [2, 3])
@pytest.mark.parametrize("kind", KINDS)
def test_regularizers(D, kind):
    pb, cp, cpw = make_problem(D, kind, seed=31)
    ev = GpuKernelEvaluator(pb)
    orc = O.Oracle(pb)
    ev.SetRegularizerRKHS(0.3)
    ev.SetRegularizerRD(0.2, 1.0)
    ev.SetRegularizerPG(0.1, 0.7)
    orc.set_regularizers(0.3, 0.2, 1.0, 0.1, 0.7)
    r, g = ev.getValueAndDerivative(abi.NCC, cp, cpw)
    ro, go = orc.evaluate(abi.NCC, cp, cpw)
    for k in ("measure", "reg_value_rkhs", "reg_value_rd", "reg_value_pg"):
        assert rel_err(r[k], ro[k]) <= TOL_VALUE, k
    assert max_rel(g, go) <= TOL_DERIV


@pytest.mark.parametrize("D", [2, 3])
@pytest.mark.parametrize("kind", ["stationary", "weight_image"])
def test_lcc(D, kind):
    shape = (10, 11, 12) if D == 3 else (24, 26)
    pb, cp, cpw = make_problem(D, kind, subsample=2, nbh=2, shape=shape, seed=41, sigma_c4=3.0, sigma_c0=6.0,
                               cp_spacing=1.5)
    ev = GpuKernelEvaluator(pb)
    orc = O.Oracle(pb)
    r, g = ev.getValueAndDerivative(abi.LCC, cp, cpw)
    ro, go = orc.evaluate(abi.LCC, cp, cpw)
    assert r["num_pixels_counted"] == ro["num_pixels_counted"]
    assert rel_err(r["measure"], ro["measure"]) <= TOL_VALUE
    assert max_rel(g, go) <= TOL_DERIV


@pytest.mark.parametrize("D", [2, 3])
def test_metric_level(D):
    pb, cp, cpw = make_problem(D, seed=51)
    params = np.ascontiguousarray(cp.T.reshape(-1))
    params[::7] = 0.0                                   # exercise the zero-parameter subgradient branches
    ev = GpuKernelEvaluator(pb)
    orc = O.Oracle(pb)
    for m in (MetricDesc.make("ncc", l1=1e-3, l21=2e-3, l2=1e-3, rd=1e-2),
              MetricDesc.make("mse", l1=5e-4, rkhs=1e-2, pg=1e-3, pg_scaling=0.5)):
        v, g = ev.metric(m, params, cpw)
        vo, go = orc.metric(m, params, cpw)
        for k in ("value", "measure", "reg_value", "reg_l1", "reg_l21", "reg_l2"):
            assert rel_err(v[k], vo[k]) <= TOL_VALUE, k
        assert max_rel(g, go) <= TOL_DERIV


def test_bspline_prefilter_gpu():
    rng = np.random.default_rng(3)
    for shape in [(9, 10, 11), (13, 17)]:
        img = rng.uniform(0, 1, shape)
        np.testing.assert_allclose(bspline_coefficients(img), O.bspline_coefficients(img), rtol=0, atol=1e-12)


def test_deterministic():
    pb, cp, cpw = make_problem(3, seed=61)
    ev = GpuKernelEvaluator(pb)
    ev.SetRegularizerRD(1e-2)
    r1, g1 = ev.getValueAndDerivative(abi.NCC, cp, cpw)
    r2, g2 = ev.getValueAndDerivative(abi.NCC, cp, cpw)
    assert r1 == r2
    assert np.array_equal(g1, g2)


@pytest.mark.parametrize("D", [2, 3])
def test_optimizer_matches_oracle(D):
    pb, _, cpw = make_problem(D, seed=71, weights=False)
    P = pb.num_parameters
    m = MetricDesc.make("ncc", rd=1e-3)
    o = OptimizerDesc.make(a=2.0, number_of_iterations=6)
    ev = GpuKernelEvaluator(pb)
    opt = Optimizer(ev, o, m, np.zeros(P), cpw)
    oo = O.OracleOptimizer(O.Oracle(pb), o, m, np.zeros(P), cpw)
    for it in range(3):
        opt.run(2)
        vals = oo.run(2)
        st = opt.state()
        assert st["iteration"] == oo.state.iteration
        assert rel_err(st["value"], vals[-1]) <= 1e-4
        assert rel_err(st["current_time"], oo.state.current_time) <= 1e-3 or abs(oo.state.current_time) < 1e-9
        assert max_rel(opt.parameters(), oo.position) <= 1e-3
    assert max_rel(opt.parameters(best=True), oo.best) <= 1e-3


# ---- phase-table path (stationary kernel, control spacing = h * fixed spacing, subsample 1) ----
TABLE_CASES = [
    # D, h, shape, sigma_c4, sigma_c0
    (3, 2, (14, 16, 18), 4.5, 9.0),
    (3, 4, (20, 22, 26), 9.0, 18.0),
    (2, 4, (40, 44), 9.0, 18.0),
    (2, 8, (48, 56), 16.0, 32.0),
]


def _table_problem(D, h, shape, s4, s0, seed, **kw):
    return make_problem(D, "stationary", shape=shape, seed=seed, sigma_c4=s4, sigma_c0=s0, cp_spacing=float(h),
                        spacing=(1.0,) * D, origin=tuple([0.5, -1.0, 2.0][:D]), **kw)


# GEMM engine of the table path: (path request, expected active path)
ENGINES = {
    "tensor": (GpuKernelEvaluator.AUTO, GpuKernelEvaluator.TABLE_TC),
    "cuda": (GpuKernelEvaluator.REQ_TABLE_CUDA_CORES, GpuKernelEvaluator.TABLE),
}


@pytest.mark.parametrize("engine", sorted(ENGINES))
@pytest.mark.parametrize("case", TABLE_CASES)
@pytest.mark.parametrize("metric", [abi.MSE, abi.NCC])
@pytest.mark.parametrize("with_df", [False, True])
def test_table_path_matches_oracle_and_generic(case, metric, with_df, engine):
    D, h, shape, s4, s0 = case
    pb, cp, cpw = _table_problem(D, h, shape, s4, s0, seed=91)
    df = _df_for(pb, 9) if with_df else None
    ev = GpuKernelEvaluator(pb)
    request, expected = ENGINES[engine]
    assert ev.path(request) == expected
    ev.SetRegularizerRD(0.05)
    ev.SetRegularizerRKHS(0.02)
    r, g = ev.getValueAndDerivative(metric, cp, cpw, df)
    orc = O.Oracle(pb)
    orc.set_regularizers(rkhs=0.02, rd=0.05)
    ro, go = orc.evaluate(metric, cp, cpw, df)
    assert r["num_pixels_counted"] == ro["num_pixels_counted"]
    for k in ("measure", "reg_value_rd", "reg_value_rkhs"):
        assert rel_err(r[k], ro[k]) <= TOL_VALUE, k
    assert max_rel(g, go) <= TOL_DERIV
    assert ev.path(1) == GpuKernelEvaluator.GENERIC
    r2, g2 = ev.getValueAndDerivative(metric, cp, cpw, df)
    assert r2["num_pixels_counted"] == r["num_pixels_counted"]
    assert rel_err(r["measure"], r2["measure"]) <= TOL_VALUE
    assert max_rel(g, g2) <= TOL_DERIV


@pytest.mark.parametrize("case", TABLE_CASES[:3])
def test_table_path_metric_level_and_optimizer(case):
    D, h, shape, s4, s0 = case
    pb, cp, cpw = _table_problem(D, h, shape, s4, s0, seed=93, weights=False)
    params = np.ascontiguousarray(cp.T.reshape(-1))
    params[::5] = 0.0
    ev = GpuKernelEvaluator(pb)
    assert ev.path() == GpuKernelEvaluator.TABLE_TC
    orc = O.Oracle(pb)
    m = MetricDesc.make("ncc", l1=1e-3, l21=1e-3, l2=1e-3, rd=1e-2, pg=1e-3)
    v, g = ev.metric(m, params, cpw)
    vo, go = orc.metric(m, params, cpw)
    for k in ("value", "measure", "reg_value"):
        assert rel_err(v[k], vo[k]) <= TOL_VALUE, k
    assert max_rel(g, go) <= TOL_DERIV
    o = OptimizerDesc.make(a=2.0, number_of_iterations=4)
    opt = Optimizer(ev, o, MetricDesc.make("ncc", rd=1e-3), np.zeros(pb.num_parameters), cpw)
    oo = O.OracleOptimizer(orc, o, MetricDesc.make("ncc", rd=1e-3), np.zeros(pb.num_parameters), cpw)
    opt.run(4)
    vals = oo.run(4)
    assert rel_err(opt.state()["value"], vals[-1]) <= 1e-4
    assert max_rel(opt.parameters(), oo.position) <= 1e-3


@pytest.mark.parametrize("orthant", [False, True])
@pytest.mark.parametrize("case", [TABLE_CASES[1], TABLE_CASES[2]])
def test_table_path_fused_step_best_parameters(case, orthant):
    """The optimizer step fused into the table gather, against the oracle optimizer and against the
    separate step kernel of the generic path: positions, best parameters read between runs (the
    pending best position of an improving step is taken over when read), best value, time."""
    D, h, shape, s4, s0 = case
    pb, cp, cpw = _table_problem(D, h, shape, s4, s0, seed=57, weights=False)
    P = pb.num_parameters
    m = MetricDesc.make("ncc", rd=1e-3, l1=1e-4 if orthant else 0.0)
    o = OptimizerDesc.make(a=2.0, number_of_iterations=9, orthant_projection=orthant)
    start = np.ascontiguousarray(cp.T.reshape(-1)) * 0.5
    ev = GpuKernelEvaluator(pb)
    assert ev.path() == GpuKernelEvaluator.TABLE_TC
    opt = Optimizer(ev, o, m, start, cpw)
    ev_generic = GpuKernelEvaluator(pb)
    assert ev_generic.path(GpuKernelEvaluator.REQ_GENERIC) == GpuKernelEvaluator.GENERIC
    opt_generic = Optimizer(ev_generic, o, m, start, cpw)
    oo = O.OracleOptimizer(O.Oracle(pb), o, m, start, cpw)
    for chunk in (1, 3, 2, 3):
        opt.run(chunk)
        opt_generic.run(chunk)
        oo.run(chunk)
        st, sg = opt.state(), opt_generic.state()
        assert st["iteration"] == sg["iteration"] == oo.state.iteration
        assert rel_err(st["best_value"], oo.state.best_value) <= 1e-4
        assert rel_err(st["best_value"], sg["best_value"]) <= 1e-4
        assert max_rel(opt.parameters(), oo.position) <= 1e-3
        assert max_rel(opt.parameters(best=True), oo.best) <= 1e-3
        assert max_rel(opt.parameters(best=True), opt_generic.parameters(best=True)) <= 1e-3


# LCC with the anisotropic (weight-tensor) kernel: the 3-D derivative keeps the reference's
# form (neighbour covariance at both ends of k(c_i, n), no control-point weight w_i;
# GpuEvaluatorLCC.cu:206-530), so the weights are random here and still must match
@pytest.mark.parametrize("D,shape,cp_spacing", [(2, (48, 52), 1.5), (3, (20, 21, 22), 2.0)])
@pytest.mark.parametrize("kind", ["weight_tensor", "weight_image"])
def test_lcc_nonstationary_larger(D, shape, cp_spacing, kind):
    pb, cp, cpw = make_problem(D, kind, subsample=2, nbh=2, shape=shape, seed=43, sigma_c4=3.0, sigma_c0=6.0,
                               cp_spacing=cp_spacing)
    ev = GpuKernelEvaluator(pb)
    orc = O.Oracle(pb)
    for call in range(2):                               # the second call redraws the sample shifts
        r, g = ev.getValueAndDerivative(abi.LCC, cp, cpw)
        ro, go = orc.evaluate(abi.LCC, cp, cpw)
        assert r["num_pixels_counted"] == ro["num_pixels_counted"]
        assert rel_err(r["measure"], ro["measure"]) <= TOL_VALUE
        assert max_rel(g, go) <= TOL_DERIV


@pytest.mark.parametrize("D,kind", [(2, "stationary"), (3, "weight_tensor")])
def test_optimizer_lcc_matches_oracle(D, kind):
    """The device optimizer with LCC (its dense fields allocated before the iteration is captured)
    against the FP64 oracle optimizer, with RKHS + L1 as in the CT-like workload."""
    shape = (12, 13, 14) if D == 3 else (28, 30)
    pb, _, cpw = make_problem(D, kind, subsample=2, nbh=2, shape=shape, seed=73, sigma_c4=3.0, sigma_c0=6.0,
                              cp_spacing=1.5, weights=False)
    P = pb.num_parameters
    m = MetricDesc.make("lcc", rkhs=1e-3, l1=1e-4)
    o = OptimizerDesc.make(a=5.0, number_of_iterations=4)
    ev = GpuKernelEvaluator(pb)
    opt = Optimizer(ev, o, m, np.zeros(P), cpw)
    oo = O.OracleOptimizer(O.Oracle(pb), o, m, np.zeros(P), cpw)
    opt.run(4)
    vals = oo.run(4)
    st = opt.state()
    assert st["iteration"] == 4
    assert rel_err(st["value"], vals[-1]) <= 1e-4
    assert max_rel(opt.parameters(), oo.position) <= 1e-3


def test_metric_with_page_locked_caller_buffers_matches_pageable():
    """skm_metric_evaluate reads page-locked parameters and writes a page-locked derivative directly
    (no staging copies); the results equal those of ordinary host arrays bit for bit."""
    torch = pytest.importorskip("torch")
    pb, cp, cpw = make_problem(3, seed=77)
    params = np.ascontiguousarray(cp.T.reshape(-1))
    m = MetricDesc.make("ncc", rd=1e-2, l1=1e-4)
    ev = GpuKernelEvaluator(pb)
    v0, g0 = ev.metric(m, params, cpw)
    pp = torch.zeros(params.size, dtype=torch.float64, pin_memory=True).numpy()
    gp = torch.zeros(params.size, dtype=torch.float64, pin_memory=True).numpy()
    for scale in (1.0, 0.5):                        # two calls: the graph keyed by the buffers is replayed
        pp[:] = params * scale
        v1, _ = ev.metric(m, pp, cpw, out_derivative=gp)
        v2, g2 = ev.metric(m, params * scale, cpw)
        assert v1 == v2 and np.array_equal(gp, g2)
    assert v0["value"] == ev.metric(m, params, cpw)[0]["value"]
    # two derivative buffers used alternately (each keeps its graph in the evaluator's cache)
    g_alt = [gp, torch.zeros(params.size, dtype=torch.float64, pin_memory=True).numpy()]
    for i, scale in enumerate((0.9, 0.8, 0.7, 0.6, 0.5)):
        pp[:] = params * scale
        ev.metric(m, pp, cpw, out_derivative=g_alt[i & 1])
        _, g2 = ev.metric(m, params * scale, cpw)
        assert np.array_equal(g_alt[i & 1], g2)
