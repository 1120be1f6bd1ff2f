"""ctypes front end of the test-side checkers in this directory.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py.  Wraps
  * the FP64 oracle (skm_oracle.c -> _build/libskm_oracle.so),
  * the reference's host-compiled math headers (_ref/libskmref_host_d{2,3}.so),
  * the reference's own CUDA evaluator (_ref/libskmref_gpu_*.so), when built.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from skmimageregistration_b200.abi import (EvaluatorDesc, Field, Geometry, MetricDesc,
                                           MetricValues, OptimizerDesc, Result, dptr, field)
from skmimageregistration_b200.problem import Problem

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libskm_oracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


def build_oracle():
    """Compile the oracle (gcc) if its library is missing or stale."""
    src = os.path.join(HERE, "skm_oracle.c")
    if not os.path.exists(ORACLE_SO) or os.path.getmtime(ORACLE_SO) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", HERE, "oracle"])
    return ORACLE_SO


class OptState(C.Structure):
    _fields_ = [("iteration", C.c_int32), ("current_time", C.c_double), ("learning_rate", C.c_double),
                ("scalar_product", C.c_double), ("best_value", C.c_double), ("last_value", C.c_double)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build_oracle())
        L = _lib
        L.ora_create.restype = C.c_void_p
        L.ora_create.argtypes = [C.POINTER(EvaluatorDesc)]
        L.ora_destroy.argtypes = [C.c_void_p]
        L.ora_set_regularizers.argtypes = [C.c_void_p] + [C.c_double] * 5
        L.ora_evaluate.argtypes = [C.c_void_p, C.c_int, _dp, _dp, C.POINTER(Field), C.c_int, _dp,
                                   C.POINTER(Result)]
        L.ora_displacement_field.argtypes = [C.c_void_p, _dp, _dp, C.POINTER(Field), _dp]
        L.ora_metric_evaluate.argtypes = [C.c_void_p, C.POINTER(MetricDesc), _dp, _dp, C.POINTER(Field),
                                          _dp, C.POINTER(MetricValues)]
        L.ora_optimize.argtypes = [C.c_void_p, C.POINTER(OptimizerDesc), C.POINTER(MetricDesc), _dp,
                                   C.POINTER(Field), C.c_int, _dp, _dp, _dp, _dp, C.POINTER(OptState), _dp]
        L.ora_bspline_coefficients.argtypes = [C.c_int, _ip, _dp, _dp]
        L.ora_bspline_sample.argtypes = [C.c_int, _dp, C.POINTER(Geometry), C.c_int64, _dp, _ip, _dp, _dp]
        L.ora_kernel_values.argtypes = [C.POINTER(EvaluatorDesc), C.c_int64, _dp, _dp, _dp]
        L.ora_pcg32_shifts.argtypes = [C.POINTER(C.c_uint64), C.c_int64, C.c_int, C.c_int, _ip]
        L.ora_pcg32_next.restype = C.c_uint32
        L.ora_pcg32_next.argtypes = [C.POINTER(C.c_uint64)]
        L.ora_last_shifts.restype = _ip
        L.ora_last_shifts.argtypes = [C.c_void_p]
        L.ora_num_subsampled.restype = C.c_int64
        L.ora_num_subsampled.argtypes = [C.c_void_p]
        L.ora_set_num_threads.argtypes = [C.c_int]
    return _lib


def set_num_threads(n):
    lib().ora_set_num_threads(int(n))


def bspline_coefficients(image):
    """BsplineImage::computeCoeffs restated (FP64)."""
    img = np.ascontiguousarray(image, dtype=np.float64)
    D = img.ndim
    size = (C.c_int32 * 3)(*(list(reversed(img.shape)) + [1] * (3 - D)))
    out = np.zeros(tuple(s + 3 for s in img.shape), dtype=np.float64)
    lib().ora_bspline_coefficients(D, size, dptr(img), dptr(out))
    return out


def bspline_sample(coeffs, geometry, points):
    D = coeffs.ndim
    pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, D)
    n = pts.shape[0]
    inside = np.zeros(n, np.int32)
    vals = np.zeros(n)
    grads = np.zeros((n, D))
    lib().ora_bspline_sample(D, dptr(np.ascontiguousarray(coeffs, np.float64)), C.byref(geometry), n,
                             dptr(pts), inside.ctypes.data_as(_ip), dptr(vals), dptr(grads))
    return inside, vals, grads


def kernel_values(desc, p, q):
    D = desc.dimensions
    p = np.ascontiguousarray(p, np.float64).reshape(-1, D)
    q = np.ascontiguousarray(q, np.float64).reshape(-1, D)
    k = np.zeros(p.shape[0])
    lib().ora_kernel_values(C.byref(desc), p.shape[0], dptr(p), dptr(q), dptr(k))
    return k


def pcg32_shifts(n, D, subsample, state=0xBA5EBA11DEADBEEF):
    st = C.c_uint64(state)
    out = np.zeros((n, D), np.int32)
    lib().ora_pcg32_shifts(C.byref(st), n, D, subsample, out.ctypes.data_as(_ip))
    return out, st.value


class Oracle:
    """FP64 restatement of one GpuKernelEvaluator (same call pattern)."""

    def __init__(self, problem: Problem):
        self.problem = problem
        self._desc = problem.desc()
        self.h = lib().ora_create(C.byref(self._desc))
        self.D = problem.D

    def close(self):
        if self.h:
            lib().ora_destroy(self.h)
            self.h = None

    __del__ = close

    def set_regularizers(self, rkhs=0.0, rd=0.0, rd_scaling=1.0, pg=0.0, pg_scaling=1.0):
        lib().ora_set_regularizers(self.h, rkhs, rd, rd_scaling, pg, pg_scaling)

    def _df(self, df, df_geometry):
        return field(df, df_geometry if df_geometry is not None else self.problem.fixed_geometry())

    def evaluate(self, metric, cp, cpw, df=None, df_geometry=None, derivative=True, do_resampling=True):
        cp = np.ascontiguousarray(cp, np.float64)
        cpw = np.ascontiguousarray(cpw, np.float64)
        f = self._df(df, df_geometry)
        res = Result()
        der = np.zeros(self.problem.num_parameters) if derivative else None
        rc = lib().ora_evaluate(self.h, metric, dptr(cp), dptr(cpw), C.byref(f), int(do_resampling),
                                dptr(der), C.byref(res))
        if rc != 0:
            raise RuntimeError("oracle: sample outside the fixed image (reference would read out of bounds)")
        return res.as_dict(), der

    def displacement_field(self, cp, cpw, df=None, df_geometry=None):
        cp = np.ascontiguousarray(cp, np.float64)
        cpw = np.ascontiguousarray(cpw, np.float64)
        f = self._df(df, df_geometry)
        out = np.zeros((self.problem.n_texels, self.D))
        lib().ora_displacement_field(self.h, dptr(cp), dptr(cpw), C.byref(f), dptr(out))
        return out

    def metric(self, mdesc, params, cpw, df=None, df_geometry=None, derivative=True):
        params = np.ascontiguousarray(params, np.float64)
        cpw = np.ascontiguousarray(cpw, np.float64)
        f = self._df(df, df_geometry)
        out = MetricValues()
        der = np.zeros(self.problem.num_parameters) if derivative else None
        lib().ora_metric_evaluate(self.h, C.byref(mdesc), dptr(params), dptr(cpw), C.byref(f), dptr(der),
                                  C.byref(out))
        return out.as_dict(), der

    def last_shifts(self):
        p = lib().ora_last_shifts(self.h)
        if not p:
            return None
        n = lib().ora_num_subsampled(self.h)
        return np.ctypeslib.as_array(p, shape=(n * self.D,)).reshape(n, self.D).copy()


class OracleOptimizer:
    """Adaptive-step gradient descent in the ITK v4 loop, FP64."""

    def __init__(self, oracle: Oracle, odesc, mdesc, initial, cpw, df=None, df_geometry=None):
        self.o = oracle
        self.odesc, self.mdesc = odesc, mdesc
        P = oracle.problem.num_parameters
        self.position = np.ascontiguousarray(initial, np.float64).copy()
        self.tmp = np.zeros(P)
        self.base = np.zeros(P)        # ITK m_PreviousGradient starts zero-filled
        self.best = self.position.copy()
        self.cpw = np.ascontiguousarray(cpw, np.float64)
        self.df = df
        self.df_geometry = df_geometry
        self.state = OptState()
        self.state.best_value = np.finfo(np.float64).max

    def run(self, iterations):
        vals = np.zeros(iterations)
        f = self.o._df(self.df, self.df_geometry)
        lib().ora_optimize(self.o.h, C.byref(self.odesc), C.byref(self.mdesc), dptr(self.cpw), C.byref(f),
                           iterations, dptr(self.position), dptr(self.tmp), dptr(self.base), dptr(self.best),
                           C.byref(self.state), dptr(vals))
        return vals


# ---------------------------------------------------------------------------------------------
# the reference itself (built by `make ref` from the reference checkout into _ref/)

def ref_host(D):
    """Host-compiled reference headers (known-answer driver) or None if not built."""
    path = os.path.join(REF_DIR, "libskmref_host_d%d.so" % D)
    if not os.path.exists(path):
        return None
    L = C.CDLL(path)
    L.skmref_bspline_coefficients.argtypes = [_ip, _dp, _dp]
    L.skmref_bspline_sample.argtypes = [_dp, C.POINTER(Geometry), C.c_int64, _dp, _ip, _dp, _dp]
    L.skmref_kernel_values.argtypes = [C.POINTER(EvaluatorDesc), C.c_int64, _dp, _dp, _dp]
    L.skmref_max_eigenvalue.restype = C.c_double
    L.skmref_max_eigenvalue.argtypes = [_dp]
    L.skmref_rng_stream.argtypes = [C.c_int64, C.POINTER(C.c_uint32)]
    L.skmref_grid_shifts.argtypes = [C.c_int64, C.c_int, _ip]
    return L


def ref_gpu_path(D, double=True, ieee=False):
    """ieee=True: the double build with IEEE arithmetic (no fast math, no multiply-add contraction)."""
    return os.path.join(REF_DIR, "libskmref_gpu_%s%d%s.so" % ("d" if double else "f", D, "_ieee" if ieee else ""))


class RefGpu:
    """The reference's own GpuKernelEvaluator (needs a GPU and the _ref build)."""

    def __init__(self, problem: Problem, double=True, ieee=False):
        path = ref_gpu_path(problem.D, double, ieee)
        L = C.CDLL(path)
        L.skmref_create.argtypes = [C.POINTER(EvaluatorDesc), C.POINTER(C.c_void_p)]
        L.skmref_destroy.argtypes = [C.c_void_p]
        L.skmref_set_regularizers.argtypes = [C.c_void_p] + [C.c_double] * 5
        L.skmref_evaluate.argtypes = [C.c_void_p, C.c_int, _dp, _dp, C.POINTER(Field), C.c_int, _dp,
                                      C.POINTER(Result)]
        L.skmref_displacement_field.argtypes = [C.c_void_p, _dp, _dp, C.POINTER(Field), _dp, C.c_int64]
        self.L = L
        self.problem = problem
        self._desc = problem.desc()
        h = C.c_void_p()
        if L.skmref_create(C.byref(self._desc), C.byref(h)) != 0:
            raise RuntimeError("reference evaluator: dimension mismatch")
        self.h = h

    def close(self):
        if self.h:
            self.L.skmref_destroy(self.h)
            self.h = None

    __del__ = close

    def set_regularizers(self, rkhs=0.0, rd=0.0, rd_scaling=1.0, pg=0.0, pg_scaling=1.0):
        self.L.skmref_set_regularizers(self.h, rkhs, rd, rd_scaling, pg, pg_scaling)

    def evaluate(self, metric, cp, cpw, df=None, df_geometry=None, derivative=True, do_resampling=True):
        cp = np.ascontiguousarray(cp, np.float64)
        cpw = np.ascontiguousarray(cpw, np.float64)
        f = field(df, df_geometry if df_geometry is not None else self.problem.fixed_geometry())
        res = Result()
        der = np.zeros(self.problem.num_parameters) if derivative else None
        rc = self.L.skmref_evaluate(self.h, metric, dptr(cp), dptr(cpw), C.byref(f), int(do_resampling),
                                    dptr(der), C.byref(res))
        if rc != 0:
            raise RuntimeError("reference evaluator refused: draw would read out of bounds")
        return res.as_dict(), der

    def displacement_field(self, cp, cpw, df=None, df_geometry=None):
        cp = np.ascontiguousarray(cp, np.float64)
        cpw = np.ascontiguousarray(cpw, np.float64)
        f = field(df, df_geometry if df_geometry is not None else self.problem.fixed_geometry())
        out = np.zeros((self.problem.n_texels, self.problem.D))
        self.L.skmref_displacement_field(self.h, dptr(cp), dptr(cpw), C.byref(f), dptr(out),
                                         self.problem.n_texels)
        return out
