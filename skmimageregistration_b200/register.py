"""Multi-scale registration (the scale loop of src/SKMReg.cxx) and its preprocessing, on the GPU.

``register(reference, target, spacing, origin, config)`` runs ``skm_register``: threshold +
rescale, then per scale level Gaussian smoothing, B-spline prefilter, control-point grid,
evaluator with the previous levels' displacement field and the device-resident adaptive-step
optimizer.  ``config`` uses the reference's option names (include/ConfigUtils.h:29-62); a list
value gives one entry per scale and its last entry repeats for later scales (the CURRENT macro,
src/SKMReg.cxx:48-49).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from .abi import Geometry, RegisterDesc, RegisterReport, dptr
from .evaluator import check, lib

# include/ConfigUtils.h:29-62, the options this driver uses; weight_filename and
# weight_tensor_filename become the weight_image / weight_tensor / guidance_image arrays of register()
DEFAULT_CONFIG = {
    "sigma_C4": [64, 32, 16],
    "sigma_C0": [128, 64, 32],
    "cp_spacing_scaler": 4.0,
    "reg_l1": [0, 0, 0],
    "reg_l21": [0, 0, 0],
    "reg_l2": [0, 0, 0],
    "reg_rkhs": [0, 0, 0],
    "reg_rd": [0, 0, 0],
    "reg_rd_scaling": [1, 1, 1],
    "reg_pg": [0, 0, 0],
    "reg_pg_scaling": [1, 1, 1],
    "num_scales": 3,
    "num_function_evaluations": [500, 500, 500],
    "initial_step_size": [0.1, 0.1, 0.1],
    "metric": "mse",
    "sampling_rate": [5, 4, 3],
    "neighborhood_sampling": [15, 12, 9],
    "intensity_thresholds": [-1500, 3500],
    "smoothing_variance": [2, 1, 0],
    "tensor_weights": [400, 200, 100],
    "restart_at": 0,
}

PER_SCALE = ["sigma_C4", "sigma_C0", "reg_l1", "reg_l21", "reg_l2", "reg_rkhs", "reg_rd", "reg_rd_scaling", "reg_pg",
             "reg_pg_scaling", "num_function_evaluations", "initial_step_size", "sampling_rate",
             "neighborhood_sampling", "smoothing_variance", "tensor_weights"]
_FIELD = {"sigma_C4": "sigma_c4", "sigma_C0": "sigma_c0"}


def current(config, option, scale):
    """config[option][min(scale, len - 1)] (src/SKMReg.cxx:48-49); scalars apply to every scale."""
    v = config[option]
    if isinstance(v, (list, tuple)):
        return v[min(scale, len(v) - 1)]
    return v


def full_config(config=None):
    c = dict(DEFAULT_CONFIG)
    if config:
        c.update(config)
    return c


def make_desc(config, D) -> RegisterDesc:
    c = full_config(config)
    n = int(c["num_scales"])
    if not 1 <= n <= abi.MAX_SCALES:
        raise ValueError("num_scales must be in [1, %d]" % abi.MAX_SCALES)
    d = RegisterDesc()
    d.dimensions = D
    d.num_scales = n
    d.metric = abi.METRICS[c["metric"]]
    d.cp_spacing_scaler = float(c["cp_spacing_scaler"])
    th = c.get("intensity_thresholds") or []
    d.restart_at = int(c.get("restart_at", 0))
    d.apply_threshold = int(len(th) == 2)
    if len(th) == 2:
        d.threshold_min, d.threshold_max = float(th[0]), float(th[1])
    for opt in PER_SCALE:
        arr = getattr(d, _FIELD.get(opt, opt))
        for s in range(abi.MAX_SCALES):
            arr[s] = current(c, opt, min(s, n - 1))
    return d


def register(reference, target, spacing=None, origin=None, config=None, guidance_image=None, weight_tensor=None,
             weight_image=None, initial_displacement=None, on_level=None, first_level_parameters=None,
             on_level_parameters=None):
    """Registers `reference` (moving) onto `target` (fixed); both arrays (Z, Y, X) or (Y, X) with
    the same geometry.  Returns (displacement (..., D) on that grid, report dict).

    Kernel weighting as src/SKMReg.cxx:245-297, all images on the same grid: per level with
    tensor_weights > 0 a covariance tensor from `guidance_image` (the reference's
    weight_tensor_filename read as an image) or, without one, from the smoothed target; with
    tensor_weights == 0 the external `weight_tensor` (..., D, D) when given; `weight_image`
    (the reference's weight_filename) takes precedence in the kernel.

    Restart (config "restart_at" > 1, src/SKMReg.cxx:96-123): `initial_displacement` (..., D) is
    the summed field after level restart_at - 1; without it every level runs.  `on_level(level,
    displacement)` is called after each level with a copy of the summed field so far (the
    df-full-<level> checkpoint of the reference).

    Learned warm start: `first_level_parameters` (planar C*D kernel weights of the first level run's
    control-point grid) replace the zero start of that level; `on_level_parameters(level, alpha)`
    receives each level's best kernel weights (the warm-start network's labels)."""
    ref = np.ascontiguousarray(reference, np.float64)
    tar = np.ascontiguousarray(target, np.float64)
    if ref.shape != tar.shape:
        raise ValueError("reference and target must share their grid")
    D = ref.ndim
    geo = Geometry.make(tuple(reversed(ref.shape)), origin, spacing)
    desc = make_desc(config, D)
    keep = []
    for name, arr, shape in (("guidance_image", guidance_image, ref.shape),
                             ("weight_tensor", weight_tensor, ref.shape + (D, D)),
                             ("weight_image", weight_image, ref.shape),
                             ("initial_displacement", initial_displacement, ref.shape + (D,))):
        if arr is not None:
            a = np.ascontiguousarray(arr, np.float64)
            if a.shape != shape:
                raise ValueError("%s must have shape %s" % (name, shape))
            keep.append(a)
            setattr(desc, name, dptr(a))
    if on_level is not None:
        def _level(level, ptr, _user):
            on_level(int(level), np.ctypeslib.as_array(ptr, shape=ref.shape + (D,)).copy())
        desc.level_done = abi.LEVEL_CALLBACK(_level)
        keep.append(desc.level_done)
    if first_level_parameters is not None:              # learned warm start of the first level run
        p0 = np.ascontiguousarray(first_level_parameters, np.float64).reshape(-1)
        keep.append(p0)
        desc.first_level_parameters = dptr(p0)
        desc.first_level_parameter_count = p0.size
    if on_level_parameters is not None:
        def _params(level, ptr, count, _user):
            on_level_parameters(int(level), np.ctypeslib.as_array(ptr, shape=(int(count),)).copy())
        desc.level_parameters = abi.PARAMS_CALLBACK(_params)
        keep.append(desc.level_parameters)
    disp = np.zeros(ref.shape + (D,))
    rep = RegisterReport()
    check(lib().skm_register(C.byref(desc), C.byref(geo), dptr(ref), dptr(tar), dptr(disp), C.byref(rep)))
    return disp, rep.as_dict()


def anisotropic_tensor(image, spacing=None, sigma=64.0, weight=400.0, alignment_direction=2):
    """ComputeAnisotropicTensor (include/AnisotropicTensorUtils.h:37-371, anisotropic_filtering
    false) on the GPU: (covariance (..., D, D), maximum tilt)."""
    img = np.ascontiguousarray(image, np.float64)
    D = img.ndim
    geo = Geometry.make(tuple(reversed(img.shape)), None, spacing)
    cov = np.empty(img.shape + (D, D))
    tilt = C.c_double(0.0)
    check(lib().skm_anisotropic_tensor(D, C.byref(geo), dptr(img), float(sigma), float(weight),
                                       int(alignment_direction), dptr(cov), C.byref(tilt)))
    return cov, tilt.value


def gaussian_smooth(image, spacing=None, variance=1.0, use_image_spacing=True, maximum_error=0.01,
                    maximum_kernel_width=64):
    """GaussianSmoothing (include/itkUtils.h:139-150) on the GPU."""
    img = np.ascontiguousarray(image, np.float64)
    geo = Geometry.make(tuple(reversed(img.shape)), None, spacing)
    out = np.empty_like(img)
    check(lib().skm_gaussian_smooth(img.ndim, C.byref(geo), float(variance), int(bool(use_image_spacing)),
                                    float(maximum_error), int(maximum_kernel_width), dptr(img), dptr(out)))
    return out


def threshold_rescale(image, thresholds=(-1500, 3500), out_range=(0.0, 1.0)):
    """ThresholdImage + RescaleImage (include/itkUtils.h:45-110) on the GPU; thresholds None: rescale only."""
    img = np.ascontiguousarray(image, np.float64)
    size = (C.c_int32 * 3)(*(list(reversed(img.shape)) + [1] * (3 - img.ndim)))
    out = np.empty_like(img)
    apply = thresholds is not None and len(thresholds) == 2
    tmin, tmax = (float(thresholds[0]), float(thresholds[1])) if apply else (0.0, 0.0)
    check(lib().skm_threshold_rescale(img.ndim, size, int(apply), tmin, tmax, float(out_range[0]),
                                      float(out_range[1]), dptr(img), dptr(out)))
    return out


def warp_image(image, displacement, image_spacing=None, image_origin=None, field_spacing=None, field_origin=None,
               order=3, default_value=0.0):
    """I(p + u(p)) on the displacement field's grid (WarpImage, include/itkUtils.h:163-178, order 3;
    the final resampling of src/SKMReg.cxx:504-522, order 1) on the GPU."""
    img = np.ascontiguousarray(image, np.float64)
    u = np.ascontiguousarray(displacement, np.float64)
    D = img.ndim
    if u.ndim != D + 1 or u.shape[-1] != D:
        raise ValueError("displacement must have shape (..., %d)" % D)
    gi = Geometry.make(tuple(reversed(img.shape)), image_origin, image_spacing)
    gf = Geometry.make(tuple(reversed(u.shape[:-1])), field_origin if field_origin is not None else image_origin,
                       field_spacing if field_spacing is not None else image_spacing)
    out = np.empty(u.shape[:-1])
    check(lib().skm_warp_image(D, C.byref(gi), dptr(img), C.byref(gf), dptr(u), int(order), float(default_value),
                               dptr(out)))
    return out


def jacobian_determinant(field, spacing=None):
    """JacobianDeterminant (include/itkUtils.h:153-161) of a (..., D) vector field on the GPU."""
    u = np.ascontiguousarray(field, np.float64)
    D = u.ndim - 1
    if D not in (2, 3) or u.shape[-1] != D:
        raise ValueError("field must have shape (Y, X, 2) or (Z, Y, X, 3)")
    geo = Geometry.make(tuple(reversed(u.shape[:-1])), None, spacing)
    out = np.empty(u.shape[:-1])
    check(lib().skm_jacobian_determinant(D, C.byref(geo), dptr(u), dptr(out)))
    return out
