"""Host-side mirror of the reference's evaluator interface over the C-ABI.

``GpuKernelEvaluator`` keeps the names, argument meaning and call order of the
reference class (include/cuda/GpuEvaluator.h:69-179): construct once per scale
level, set the regularizers, then call ``getValue`` / ``getValueAndDerivative`` /
``evaluateDisplacementField`` with the current control points.  ``Metric`` and
``Optimizer`` mirror the ITK glue that drives it
(itkRegularizedImageToImageMetricv4.hxx, itkAdaptiveStepGradientDescentOptimizerv4.hxx).

Every call goes through the CUDA library (skmimageregistration_b200/_lib/libskm_b200.so);
there is no CPU fallback.  If the library is missing, importing works but the
first use raises ``SkmError``.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import abi
from .abi import (EvaluatorDesc, EvaluatorInfo, Field, MetricDesc, MetricValues, OptimizerDesc, OptimizerState, Result,
                  dptr, field)
from .problem import Problem, aos_to_flat, flat_to_aos

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib", "libskm_b200.so")

_dp = C.POINTER(C.c_double)
_lib = None


class SkmError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("skm error %d: %s" % (code, msg))
        self.code = code


def lib():
    """The loaded CUDA library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise SkmError(abi.SKM_ERR_STATE, "CUDA library %s not built (run skmimageregistration_b200/build.py)"
                           % LIB_PATH)
        L = C.CDLL(LIB_PATH)
        L.skm_last_error.restype = C.c_char_p
        L.skm_abi_version.restype = C.c_int32
        L.skm_evaluator_create.argtypes = [C.POINTER(EvaluatorDesc), C.POINTER(C.c_void_p)]
        L.skm_evaluator_destroy.argtypes = [C.c_void_p]
        L.skm_evaluator_describe.argtypes = [C.c_void_p, C.POINTER(EvaluatorInfo)]
        L.skm_evaluator_path.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.c_int32)]
        L.skm_evaluator_wait_drill.argtypes = [C.c_void_p, C.c_int32]
        L.skm_set_regularizer_rkhs.argtypes = [C.c_void_p, C.c_double]
        L.skm_set_regularizer_rd.argtypes = [C.c_void_p, C.c_double, C.c_double]
        L.skm_set_regularizer_pg.argtypes = [C.c_void_p, C.c_double, C.c_double]
        L.skm_get_value.argtypes = [C.c_void_p, C.c_int32, _dp, _dp, C.POINTER(Field), C.c_int32, C.POINTER(Result)]
        L.skm_get_value_and_derivative.argtypes = [C.c_void_p, C.c_int32, _dp, _dp, C.POINTER(Field), _dp, C.c_int32,
                                                   C.POINTER(Result)]
        L.skm_evaluate_displacement_field.argtypes = [C.c_void_p, _dp, _dp, C.POINTER(Field), _dp]
        L.skm_metric_evaluate.argtypes = [C.c_void_p, C.POINTER(MetricDesc), C.c_void_p, C.c_void_p, C.POINTER(Field),
                                          C.c_void_p,
                                          C.POINTER(MetricValues)]
        L.skm_optimizer_create.argtypes = [C.c_void_p, C.POINTER(OptimizerDesc), C.POINTER(MetricDesc), _dp, _dp,
                                           C.POINTER(Field), C.POINTER(C.c_void_p)]
        L.skm_optimizer_run.argtypes = [C.c_void_p, C.c_int32]
        L.skm_optimizer_enqueue.argtypes = [C.c_void_p, C.c_int32, C.c_void_p]
        L.skm_optimizer_profile.argtypes = [C.c_void_p, C.c_int32, _dp, C.c_int32]
        L.skm_optimizer_graph_kernel_count.argtypes = [C.c_void_p, C.POINTER(C.c_int32)]
        L.skm_optimizer_get_parameters.argtypes = [C.c_void_p, C.c_int32, _dp]
        L.skm_optimizer_get_state.argtypes = [C.c_void_p, C.POINTER(OptimizerState)]
        L.skm_optimizer_destroy.argtypes = [C.c_void_p]
        L.skm_bspline_coefficients.argtypes = [C.c_int32, C.POINTER(C.c_int32), _dp, _dp]
        L.skm_gaussian_smooth.argtypes = [C.c_int32, C.POINTER(abi.Geometry), C.c_double, C.c_int32, C.c_double,
                                          C.c_int32, _dp, _dp]
        L.skm_threshold_rescale.argtypes = [C.c_int32, C.POINTER(C.c_int32), C.c_int32, C.c_double, C.c_double,
                                            C.c_double, C.c_double, _dp, _dp]
        L.skm_register.argtypes = [C.POINTER(abi.RegisterDesc), C.POINTER(abi.Geometry), _dp, _dp, _dp,
                                   C.POINTER(abi.RegisterReport)]
        L.skm_anisotropic_tensor.argtypes = [C.c_int32, C.POINTER(abi.Geometry), _dp, C.c_double, C.c_double,
                                             C.c_int32, _dp, _dp]
        L.skm_warp_image.argtypes = [C.c_int32, C.POINTER(abi.Geometry), _dp, C.POINTER(abi.Geometry), _dp, C.c_int32,
                                     C.c_double, _dp]
        L.skm_jacobian_determinant.argtypes = [C.c_int32, C.POINTER(abi.Geometry), _dp, _dp]
        L.skm_batch_create.argtypes = [C.c_int32, C.POINTER(abi.BatchPair), C.POINTER(C.c_void_p)]
        L.skm_batch_destroy.argtypes = [C.c_void_p]
        L.skm_batch_evaluate.argtypes = [C.c_void_p]
        L.skm_batch_run.argtypes = [C.c_void_p, C.c_int32]
        L.skm_batch_enqueue.argtypes = [C.c_void_p, C.c_int32, C.c_void_p]
        L.skm_batch_set_parameters.argtypes = [C.c_void_p, C.c_int32, _dp, _dp]
        L.skm_batch_get_result.argtypes = [C.c_void_p, C.c_int32, C.POINTER(MetricValues), _dp]
        L.skm_batch_get_parameters.argtypes = [C.c_void_p, C.c_int32, C.c_int32, _dp]
        L.skm_batch_get_state.argtypes = [C.c_void_p, C.c_int32, C.POINTER(OptimizerState)]
        L.skm_batch_describe.argtypes = [C.c_void_p, C.POINTER(abi.BatchInfo)]
        _lib = L
    return _lib


def check(rc):
    if rc != 0:
        raise SkmError(rc, lib().skm_last_error().decode())


def bspline_coefficients(image):
    """BsplineImage::computeCoeffs on the GPU: (size+3)^D mirror-padded coefficients."""
    img = np.ascontiguousarray(image, dtype=np.float64)
    D = img.ndim
    size = (C.c_int32 * 3)(*(list(reversed(img.shape)) + [1] * (3 - D)))
    out = np.zeros(tuple(s + 3 for s in img.shape), dtype=np.float64)
    check(lib().skm_bspline_coefficients(D, size, dptr(img), dptr(out)))
    return out


class GpuKernelEvaluator:
    """Mirror of the reference class of the same name (GpuEvaluator.h:69-179).

    Control points ``cp`` are AoS (C, D) float64, weights ``cpw`` (C,), the
    derivative is planar (D*C,) like the reference's parameter layout.
    """

    MSE, NCC, LCC, LCC_BOX = abi.MSE, abi.NCC, abi.LCC, abi.LCC_BOX

    def __init__(self, problem: Problem):
        self.problem = problem
        self._desc = problem.desc()
        h = C.c_void_p()
        check(lib().skm_evaluator_create(C.byref(self._desc), C.byref(h)))
        self.h = h
        self.D = problem.D
        self.C = problem.C
        self._df_keep = None

    def close(self):
        if getattr(self, "h", None):
            lib().skm_evaluator_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    GENERIC, TABLE, TABLE_TC = 1, 2, 3
    # requests: -1 query, 0 automatic (table path, tensor-core GEMMs where they fit),
    # 1 generic kernels, 2 table path with CUDA-core GEMMs
    AUTO, REQ_GENERIC, REQ_TABLE_CUDA_CORES, REQ_TABLE_TC_BRICKS = 0, 1, 2, 3

    def path(self, request=-1):
        """Select and/or query the kernel path: returns 1 generic, 2 table, 3 table on tensor cores."""
        a = C.c_int32()
        check(lib().skm_evaluator_path(self.h, int(request), C.byref(a)))
        return a.value

    def describe(self):
        """Kernel path and the sizes that set the cost of one evaluation."""
        info = EvaluatorInfo()
        check(lib().skm_evaluator_describe(self.h, C.byref(info)))
        return info.as_dict()

    def wait_drill(self, armed=True):
        """Arm the bounded-wait drill: the next getValueAndDerivative on the tensor-core table path
        makes one wait of the contrib GEMM run out and raises SkmError(SKM_ERR_TIMEOUT)."""
        check(lib().skm_evaluator_wait_drill(self.h, int(bool(armed))))

    # --- GpuEvaluator.h:156-158
    def SetRegularizerRKHS(self, weight):
        check(lib().skm_set_regularizer_rkhs(self.h, float(weight)))

    def SetRegularizerRD(self, weight, scaling=1.0):
        check(lib().skm_set_regularizer_rd(self.h, float(weight), float(scaling)))

    def SetRegularizerPG(self, weight, scaling=1.0):
        check(lib().skm_set_regularizer_pg(self.h, float(weight), float(scaling)))

    def _field(self, df, df_geometry):
        if df is not None:
            df = np.ascontiguousarray(df, np.float64)
            self._df_keep = df
        return field(df, df_geometry if df_geometry is not None else self.problem.fixed_geometry())

    # --- GpuEvaluator.h:162-173
    def getValue(self, metric, cp, cpw, df=None, df_geometry=None, do_resampling=True):
        cp = np.ascontiguousarray(cp, np.float64)
        cpw = np.ascontiguousarray(cpw, np.float64)
        f = self._field(df, df_geometry)
        r = Result()
        check(lib().skm_get_value(self.h, int(metric), dptr(cp), dptr(cpw), C.byref(f), int(do_resampling),
                                  C.byref(r)))
        return r.as_dict()

    def getValueAndDerivative(self, metric, cp, cpw, df=None, df_geometry=None, derivatives=None,
                              do_resampling=True):
        cp = np.ascontiguousarray(cp, np.float64)
        cpw = np.ascontiguousarray(cpw, np.float64)
        f = self._field(df, df_geometry)
        if derivatives is None:
            derivatives = np.zeros(self.problem.num_parameters)
        r = Result()
        check(lib().skm_get_value_and_derivative(self.h, int(metric), dptr(cp), dptr(cpw), C.byref(f),
                                                 dptr(derivatives), int(do_resampling), C.byref(r)))
        return r.as_dict(), derivatives

    # --- GpuEvaluator.h:175-178
    def evaluateDisplacementField(self, cp, cpw, df=None, df_geometry=None):
        cp = np.ascontiguousarray(cp, np.float64)
        cpw = np.ascontiguousarray(cpw, np.float64)
        f = self._field(df, df_geometry)
        out = np.zeros((self.problem.n_texels, self.D))
        check(lib().skm_evaluate_displacement_field(self.h, dptr(cp), dptr(cpw), C.byref(f), dptr(out)))
        return out

    # --- metric level (RegularizedImageToImageMetricv4::GetValueAndDerivative)
    def metric(self, mdesc: MetricDesc, params, cpw, df=None, df_geometry=None, derivative=True, out_derivative=None):
        """Metric value and (negated, regularized) derivative; `out_derivative` (float64, contiguous,
        num_parameters) receives the derivative in place of a new array."""
        params = np.ascontiguousarray(params, np.float64)
        cpw = np.ascontiguousarray(cpw, np.float64)
        if df is None and df_geometry is None:           # the common call: no field, one cached struct
            f = self.__dict__.get("_nofield")
            if f is None:
                f = self._nofield = self._field(None, None)
        else:
            f = self._field(df, df_geometry)
        out = MetricValues()
        if not derivative:
            der = None
        elif out_derivative is not None:
            der = out_derivative
            assert der.dtype == np.float64 and der.flags["C_CONTIGUOUS"] and der.size == self.problem.num_parameters
        else:
            der = np.zeros(self.problem.num_parameters)
        check(lib().skm_metric_evaluate(self.h, C.byref(mdesc), params.ctypes.data, cpw.ctypes.data, C.byref(f),
                                        der.ctypes.data if der is not None else None, C.byref(out)))
        return out.as_dict(), der


class Optimizer:
    """Device-resident AdaptiveStepGradientDescentOptimizerv4 (one CUDA graph per iteration)."""

    def __init__(self, evaluator: GpuKernelEvaluator, odesc: OptimizerDesc, mdesc: MetricDesc, initial, cpw,
                 df=None, df_geometry=None):
        self.ev = evaluator
        self.odesc, self.mdesc = odesc, mdesc
        init = np.ascontiguousarray(initial, np.float64)
        cpw = np.ascontiguousarray(cpw, np.float64)
        f = evaluator._field(df, df_geometry)
        h = C.c_void_p()
        check(lib().skm_optimizer_create(evaluator.h, C.byref(odesc), C.byref(mdesc), dptr(init), dptr(cpw),
                                         C.byref(f), C.byref(h)))
        self.h = h

    def run(self, iterations):
        check(lib().skm_optimizer_run(self.h, int(iterations)))

    def enqueue(self, iterations):
        """Enqueue iterations without waiting; returns the CUDA stream handle (int)."""
        s = C.c_void_p()
        check(lib().skm_optimizer_enqueue(self.h, int(iterations), C.byref(s)))
        return s.value

    PHASES = ("pack", "shifts", "transform", "warp", "stats", "contrib", "gather", "result", "update")

    def profile(self, iterations):
        """Mean milliseconds per phase over `iterations` un-graphed iterations."""
        out = np.zeros(9)
        check(lib().skm_optimizer_profile(self.h, int(iterations), dptr(out), 9))
        return dict(zip(self.PHASES, out.tolist()))

    def graph_kernel_count(self):
        n = C.c_int32()
        check(lib().skm_optimizer_graph_kernel_count(self.h, C.byref(n)))
        return n.value

    def parameters(self, best=False):
        out = np.zeros(self.ev.problem.num_parameters)
        check(lib().skm_optimizer_get_parameters(self.h, int(bool(best)), dptr(out)))
        return out

    def state(self):
        s = OptimizerState()
        check(lib().skm_optimizer_get_state(self.h, C.byref(s)))
        return s.as_dict()

    def close(self):
        if getattr(self, "h", None):
            lib().skm_optimizer_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many registration pairs in one persistent kernel per optimizer iteration (skm_batch_*).

    problems: list of Problem; metrics / optimizers: one MetricDesc / OptimizerDesc per pair (or one
    for all); initial: planar parameters per pair (None: zeros); cpws: weights per pair (None: ones).
    """

    def __init__(self, problems, metrics, optimizers, initial=None, cpws=None):
        n = len(problems)
        metrics = metrics if isinstance(metrics, (list, tuple)) else [metrics] * n
        optimizers = optimizers if isinstance(optimizers, (list, tuple)) else [optimizers] * n
        self.problems = list(problems)
        self._descs = [pb.desc() for pb in self.problems]
        self._keep = []
        arr = (abi.BatchPair * n)()
        for i, pb in enumerate(self.problems):
            arr[i].evaluator = C.pointer(self._descs[i])
            arr[i].metric = metrics[i]
            arr[i].optimizer = optimizers[i]
            p0 = None if initial is None or initial[i] is None else np.ascontiguousarray(initial[i], np.float64)
            w0 = None if cpws is None or cpws[i] is None else np.ascontiguousarray(cpws[i], np.float64)
            self._keep += [p0, w0]
            arr[i].initial_parameters = dptr(p0)
            arr[i].cpw = dptr(w0)
        h = C.c_void_p()
        check(lib().skm_batch_create(n, arr, C.byref(h)))
        self.h = h

    def evaluate(self):
        """One value + derivative evaluation of every pair at its current parameters (no step)."""
        check(lib().skm_batch_evaluate(self.h))

    def run(self, iterations):
        check(lib().skm_batch_run(self.h, int(iterations)))

    def enqueue(self, iterations):
        """Enqueue optimizer iterations without waiting; returns the batch's cudaStream_t."""
        s = C.c_void_p()
        check(lib().skm_batch_enqueue(self.h, int(iterations), C.byref(s)))
        return s.value

    def set_parameters(self, pair, params=None, cpw=None):
        p = None if params is None else np.ascontiguousarray(params, np.float64)
        w = None if cpw is None else np.ascontiguousarray(cpw, np.float64)
        check(lib().skm_batch_set_parameters(self.h, int(pair), dptr(p), dptr(w)))

    def result(self, pair):
        v = MetricValues()
        g = np.zeros(self.problems[pair].num_parameters)
        check(lib().skm_batch_get_result(self.h, int(pair), C.byref(v), dptr(g)))
        return v.as_dict(), g

    def parameters(self, pair, best=False):
        out = np.zeros(self.problems[pair].num_parameters)
        check(lib().skm_batch_get_parameters(self.h, int(pair), int(bool(best)), dptr(out)))
        return out

    def state(self, pair):
        s = OptimizerState()
        check(lib().skm_batch_get_state(self.h, int(pair), C.byref(s)))
        return s.as_dict()

    def describe(self):
        i = abi.BatchInfo()
        check(lib().skm_batch_describe(self.h, C.byref(i)))
        return i.as_dict()

    def close(self):
        if getattr(self, "h", None):
            lib().skm_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
