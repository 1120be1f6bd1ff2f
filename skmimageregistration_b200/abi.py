"""ctypes mirror of the C-ABI in include/skm_gpu.h.

The structs here are byte-for-byte the ones declared in the header; they are
shared by the product wrapper (:mod:`skmimageregistration_b200.evaluator`) and the
test-side checkers so that both receive identical inputs.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

SKM_OK = 0
SKM_ERR_INVALID = 1
SKM_ERR_CUDA = 2
SKM_ERR_UNSUPPORTED = 3
SKM_ERR_NOMEM = 4
SKM_ERR_STATE = 5
SKM_ERR_TIMEOUT = 6

# GpuKernelEvaluator::MEASURE (include/cuda/GpuEvaluator.h:160)
MSE, NCC, LCC, LCC_BOX = 0, 1, 2, 3
METRICS = {"mse": MSE, "ncc": NCC, "lcc": LCC, "lcc_box": LCC_BOX}

_dp = C.POINTER(C.c_double)


class Geometry(C.Structure):
    """ImageBase geometry (include/cuda/ImageBase.h:40-49): origin + spacing*index."""

    _fields_ = [("origin", C.c_double * 3), ("spacing", C.c_double * 3), ("size", C.c_int32 * 3)]

    @classmethod
    def make(cls, size, origin=None, spacing=None):
        g = cls()
        D = len(size)
        origin = list(origin) if origin is not None else [0.0] * D
        spacing = list(spacing) if spacing is not None else [1.0] * D
        for d in range(3):
            g.origin[d] = float(origin[d]) if d < D else 0.0
            g.spacing[d] = float(spacing[d]) if d < D else 1.0
            g.size[d] = int(size[d]) if d < D else 1
        return g

    def dims(self, D):
        return tuple(int(self.size[d]) for d in range(D))


class Field(C.Structure):
    """ImageNearest<VecF,D> displacement field (data NULL = none)."""

    _fields_ = [("data", _dp), ("geometry", Geometry)]


class EvaluatorDesc(C.Structure):
    _fields_ = [
        ("dimensions", C.c_int32),
        ("num_parameters", C.c_int32),
        ("subsample", C.c_int32),
        ("subsample_neighborhood", C.c_int32),
        ("sigma_c0", C.c_double),
        ("sigma_c4", C.c_double),
        ("use_weight_image", C.c_int32),
        ("maximum_weight", C.c_double),
        ("weight_image", _dp),
        ("weight_image_geometry", Geometry),
        ("use_weight_tensor", C.c_int32),
        ("maximum_eigenvalue_covariance", C.c_double * 9),
        ("weight_tensor", _dp),
        ("weight_tensor_geometry", Geometry),
        ("moving_coefficients", _dp),
        ("moving_geometry", Geometry),
        ("fixed_image", _dp),
        ("fixed_geometry", Geometry),
        ("cp_geometry", Geometry),
        ("cpw_geometry", Geometry),
    ]


class Result(C.Structure):
    _fields_ = [
        ("measure", C.c_double),
        ("reg_value_rkhs", C.c_double),
        ("reg_value_rd", C.c_double),
        ("reg_value_pg", C.c_double),
        ("num_pixels_counted", C.c_uint32),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class EvaluatorInfo(C.Structure):
    _fields_ = [
        ("path", C.c_int32),
        ("dimensions", C.c_int32),
        ("fixed_texels", C.c_int64),
        ("samples", C.c_int64),
        ("control_points", C.c_int64),
        ("table_phases", C.c_int32),
        ("table_taps", C.c_int32),
        ("table_cells_per_axis", C.c_int32 * 3),
        ("table_cells", C.c_int64),
        ("table_regularizer_offsets", C.c_int32),
        ("tc_cells_per_tile", C.c_int32),
        ("tc_brick", C.c_int32 * 3),
        ("tc_transform_tiles", C.c_int64),
        ("tc_contrib_tiles", C.c_int64),
        ("tc_transform_n", C.c_int32),
        ("tc_transform_k", C.c_int32),
        ("tc_contrib_n", C.c_int32),
        ("tc_contrib_k", C.c_int32),
        ("tc_contrib_taps", C.c_int32),
        ("warp_staged", C.c_int32),
        ("tc_region_buffers", C.c_int32),
        ("tc_u_staging", C.c_int32),
        ("tc_record_slots", C.c_int32),
        ("tc_contrib_bricks", C.c_int32),
    ]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["table_cells_per_axis"] = list(self.table_cells_per_axis)
        d["tc_brick"] = list(self.tc_brick)
        return d


class MetricDesc(C.Structure):
    _fields_ = [
        ("metric", C.c_int32),
        ("reg_l1", C.c_double),
        ("reg_l21", C.c_double),
        ("reg_l2", C.c_double),
        ("reg_rkhs", C.c_double),
        ("reg_rd", C.c_double),
        ("reg_rd_scaling", C.c_double),
        ("reg_pg", C.c_double),
        ("reg_pg_scaling", C.c_double),
        ("use_negative_gradient", C.c_int32),
        ("do_resampling", C.c_int32),
    ]

    @classmethod
    def make(cls, metric="mse", l1=0.0, l21=0.0, l2=0.0, rkhs=0.0, rd=0.0, rd_scaling=1.0,
             pg=0.0, pg_scaling=1.0, use_negative_gradient=True, do_resampling=True):
        m = cls()
        m.metric = METRICS[metric] if isinstance(metric, str) else int(metric)
        m.reg_l1, m.reg_l21, m.reg_l2 = l1, l21, l2
        m.reg_rkhs, m.reg_rd, m.reg_rd_scaling = rkhs, rd, rd_scaling
        m.reg_pg, m.reg_pg_scaling = pg, pg_scaling
        m.use_negative_gradient = int(bool(use_negative_gradient))
        m.do_resampling = int(bool(do_resampling))
        return m


class MetricValues(C.Structure):
    _fields_ = [
        ("value", C.c_double),
        ("measure", C.c_double),
        ("reg_value", C.c_double),
        ("reg_l1", C.c_double),
        ("reg_l21", C.c_double),
        ("reg_l2", C.c_double),
        ("reg_rkhs", C.c_double),
        ("reg_rd", C.c_double),
        ("reg_pg", C.c_double),
        ("num_pixels_counted", C.c_uint32),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class OptimizerDesc(C.Structure):
    _fields_ = [
        ("a", C.c_double),
        ("A", C.c_double),
        ("alpha", C.c_double),
        ("f_max", C.c_double),
        ("f_min", C.c_double),
        ("omega", C.c_double),
        ("orthant_projection", C.c_int32),
        ("number_of_iterations", C.c_int32),
        ("return_best_parameters_and_value", C.c_int32),
    ]

    @classmethod
    def make(cls, a=0.1, A=20.0, alpha=1.0, f_max=1e7, f_min=-1e6, omega=1.0,
             orthant_projection=False, number_of_iterations=100, return_best=True):
        """Defaults of the reference driver (src/SKMReg.cxx:392-411)."""
        o = cls()
        o.a, o.A, o.alpha, o.f_max, o.f_min, o.omega = a, A, alpha, f_max, f_min, omega
        o.orthant_projection = int(bool(orthant_projection))
        o.number_of_iterations = int(number_of_iterations)
        o.return_best_parameters_and_value = int(bool(return_best))
        return o


class OptimizerState(C.Structure):
    _fields_ = [
        ("iteration", C.c_int32),
        ("current_time", C.c_double),
        ("learning_rate", C.c_double),
        ("value", C.c_double),
        ("best_value", C.c_double),
        ("scalar_product", C.c_double),
        ("num_pixels_counted", C.c_uint32),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


MAX_SCALES = 8


LEVEL_CALLBACK = C.CFUNCTYPE(None, C.c_int32, C.POINTER(C.c_double), C.c_void_p)
PARAMS_CALLBACK = C.CFUNCTYPE(None, C.c_int32, C.POINTER(C.c_double), C.c_int64, C.c_void_p)


class RegisterDesc(C.Structure):
    """skm_register_desc: the configuration of the reference application (src/SKMReg.cxx)."""

    _S = C.c_double * MAX_SCALES
    _I = C.c_int32 * MAX_SCALES
    _fields_ = [
        ("dimensions", C.c_int32),
        ("num_scales", C.c_int32),
        ("metric", C.c_int32),
        ("cp_spacing_scaler", C.c_double),
        ("apply_threshold", C.c_int32),
        ("threshold_min", C.c_double),
        ("threshold_max", C.c_double),
        ("sigma_c4", _S), ("sigma_c0", _S), ("smoothing_variance", _S), ("initial_step_size", _S),
        ("num_function_evaluations", _I), ("sampling_rate", _I), ("neighborhood_sampling", _I),
        ("reg_l1", _S), ("reg_l21", _S), ("reg_l2", _S), ("reg_rkhs", _S), ("reg_rd", _S),
        ("reg_rd_scaling", _S), ("reg_pg", _S), ("reg_pg_scaling", _S),
        ("tensor_weights", _S),
        ("guidance_image", C.POINTER(C.c_double)),
        ("weight_tensor", C.POINTER(C.c_double)),
        ("weight_image", C.POINTER(C.c_double)),
        ("restart_at", C.c_int32),
        ("initial_displacement", C.POINTER(C.c_double)),
        ("level_done", LEVEL_CALLBACK),
        ("level_user", C.c_void_p),
        ("first_level_parameters", C.POINTER(C.c_double)),
        ("first_level_parameter_count", C.c_int64),
        ("level_parameters", PARAMS_CALLBACK),
    ]


class RegisterReport(C.Structure):
    _fields_ = [
        ("levels_done", C.c_int32),
        ("first_level", C.c_int32),
        ("iterations", C.c_int32 * MAX_SCALES),
        ("control_points", C.c_int64 * MAX_SCALES),
        ("best_value", C.c_double * MAX_SCALES),
        ("seconds", C.c_double * MAX_SCALES),
        ("optimize_seconds", C.c_double * MAX_SCALES),
    ]

    def as_dict(self):
        n = self.levels_done
        return {"levels_done": n, "first_level": self.first_level, "iterations": list(self.iterations[:n]),
                "control_points": list(self.control_points[:n]), "best_value": list(self.best_value[:n]),
                "seconds": list(self.seconds[:n]), "optimize_seconds": list(self.optimize_seconds[:n])}


def dptr(a):
    """double* of a C-contiguous float64 numpy array (or NULL)."""
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"], "expected C-contiguous float64"
    return a.ctypes.data_as(_dp)


def field(data, geometry):
    """skm_field for a displacement field array of shape (..., D) or None."""
    f = Field()
    if data is None:
        f.data = None
        f.geometry = Geometry.make([1, 1, 1])
    else:
        f.data = dptr(data)
        f.geometry = geometry
    return f


class BatchPair(C.Structure):
    """skm_batch_pair: one pair of a batched registration."""

    _fields_ = [
        ("evaluator", C.POINTER(EvaluatorDesc)),
        ("metric", MetricDesc),
        ("optimizer", OptimizerDesc),
        ("initial_parameters", C.POINTER(C.c_double)),
        ("cpw", C.POINTER(C.c_double)),
    ]


class BatchInfo(C.Structure):
    _fields_ = [
        ("pairs", C.c_int32),
        ("fixed_texels", C.c_int64),
        ("control_points", C.c_int64),
        ("grid", C.c_int32),
        ("ctas_per_sm", C.c_int32),
        ("transform_tile", C.c_int32 * 3),
        ("warp_chunk", C.c_int32),
        ("items", C.c_int32 * 8),
        ("shared_memory", C.c_int32),
        ("tuned_ms", C.c_double),
        ("candidates", C.c_int32),
    ]

    def as_dict(self):
        out = {}
        for k, _ in self._fields_:
            v = getattr(self, k)
            out[k] = list(v) if hasattr(v, "__len__") else v
        return out
