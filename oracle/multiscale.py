"""FP64 restatements of the multi-scale driver and its preprocessing.

TEST INFRASTRUCTURE ONLY: imported by tests/ (and usable by bench.py's CPU leg), never by the
product.  Follows
  * GaussianSmoothing, include/itkUtils.h:139-150 (ITK DiscreteGaussianImageFilter: per-axis
    discrete Gaussian e^-t I_n(t), t = variance / spacing^2, grown until 1 - maximum_error of the
    mass, half width <= maximum_kernel_width, normalised; edge voxels repeated);
  * ThresholdImage + RescaleImage, include/itkUtils.h:45-110;
  * the scale loop of src/SKMReg.cxx:84-500 with the FP64 evaluator and optimizer of oracle.py.
ITK itself is not in this container: the ITK filters are restated from their published
algorithms (exact Bessel values, scipy.special.ive), so agreement with ITK is unpinned.
"""
from __future__ import annotations

import math

import numpy as np
from scipy.special import ive

from skmimageregistration_b200.abi import METRICS, MetricDesc, OptimizerDesc
from skmimageregistration_b200.problem import Problem, control_point_grid

from . import oracle as O


def gaussian_half_kernel(t, maximum_error=0.01, maximum_width=64):
    """Half kernel c[0..r] (centre first) of the discrete Gaussian of variance t (voxels)."""
    cap = 1.0 - maximum_error
    c = [float(ive(0, t)), float(ive(1, t))]
    s = c[0] + 2.0 * c[1]
    i = 2
    while s < cap:
        c.append(float(ive(i, t)))
        s += 2.0 * c[i]
        if c[i] < s * np.finfo(np.float64).eps:
            break
        if len(c) > maximum_width:
            break
        i += 1
    return np.asarray(c) / s


def gaussian_smooth(image, spacing, variance, use_image_spacing=True, maximum_error=0.01, maximum_width=64):
    """Separable discrete Gaussian, x (last numpy axis) first, edge-repeating borders, FP64."""
    out = np.asarray(image, np.float64).copy()
    D = out.ndim
    for d in range(D):                       # d = 0 is x
        ax = D - 1 - d
        sp = float(spacing[d]) if use_image_spacing else 1.0
        c = gaussian_half_kernel(variance / (sp * sp), maximum_error, maximum_width)
        r = len(c) - 1
        n = out.shape[ax]
        idx = np.arange(n)
        res = c[0] * out
        for k in range(1, r + 1):
            lo = np.take(out, np.clip(idx - k, 0, n - 1), axis=ax)
            hi = np.take(out, np.clip(idx + k, 0, n - 1), axis=ax)
            res = res + c[k] * (lo + hi)
        out = res
    return out


def threshold_rescale(image, thresholds=(-1500, 3500), out_range=(0.0, 1.0)):
    v = np.asarray(image, np.float64)
    lo, hi = float(v.min()), float(v.max())
    if thresholds is not None and len(thresholds) == 2:
        tmin, tmax = float(thresholds[0]), float(thresholds[1])
        below, above = v[v < tmax], v[v > tmin]
        if below.size == 0 or above.size == 0 or above.min() > below.max():
            raise ValueError("no intensity inside the thresholds")
        lo, hi = float(above.min()), float(below.max())
    omin, omax = float(out_range[0]), float(out_range[1])
    if hi != lo:
        scale = (omax - omin) / (hi - lo)
    elif hi != 0.0:
        scale = (omax - omin) / hi
    else:
        scale = 0.0
    return np.clip(v, lo, hi) * scale + (omin - lo * scale)


def register(reference, target, spacing, origin, config):
    """The scale loop with the FP64 evaluator / optimizer; returns (displacement, per-level best values)."""
    from skmimageregistration_b200.register import current, full_config
    c = full_config(config)
    ref = np.asarray(reference, np.float64)
    tar = np.asarray(target, np.float64)
    D = ref.ndim
    spacing = tuple(float(s) for s in (spacing or (1.0,) * D))
    origin = tuple(float(o) for o in (origin or (0.0,) * D))
    th = c.get("intensity_thresholds") or []
    ref = threshold_rescale(ref, th if len(th) == 2 else None)
    tar = threshold_rescale(tar, th if len(th) == 2 else None)
    past = None
    best = []
    for s in range(int(c["num_scales"])):
        var = float(current(c, "smoothing_variance", s))
        ref_s = gaussian_smooth(ref, spacing, var) if var > 1e-5 else ref
        tar_s = gaussian_smooth(tar, spacing, var) if var > 1e-5 else tar
        s4, s0 = float(current(c, "sigma_C4", s)), float(current(c, "sigma_C0", s))
        smin = np.float32(min(np.float32(s4), np.float32(s0)))
        scaler = float(c["cp_spacing_scaler"])
        cps = float(smin / np.float32(1.0)) if scaler < 1 else float(smin / np.float32(scaler))
        pb = Problem(fixed=tar_s, moving_coefficients=O.bspline_coefficients(ref_s), spacing=spacing, origin=origin,
                     sigma_c0=s0, sigma_c4=s4, cp_spacing=cps, subsample=int(current(c, "sampling_rate", s)),
                     subsample_neighborhood=int(current(c, "neighborhood_sampling", s)))
        assert pb.cp_size == control_point_grid(tuple(reversed(ref.shape)), spacing, origin, cps)[0]
        regs = {k: float(current(c, "reg_" + k, s)) for k in ("l1", "l21", "l2", "rkhs", "rd", "rd_scaling", "pg",
                                                               "pg_scaling")}
        m = MetricDesc.make(c["metric"], l1=regs["l1"], l21=regs["l21"], l2=regs["l2"], rkhs=regs["rkhs"],
                            rd=regs["rd"], rd_scaling=regs["rd_scaling"], pg=regs["pg"], pg_scaling=regs["pg_scaling"])
        others = [regs[k] for k in ("l2", "rkhs", "rd", "pg")]
        orthant = (regs["l1"] > 0 and regs["l21"] <= 0 and all(v <= 0 for v in others)) or \
                  (regs["l1"] <= 0 and regs["l21"] > 0 and all(v <= 0 for v in others))
        n_it = int(current(c, "num_function_evaluations", s))
        od = OptimizerDesc.make(a=float(current(c, "initial_step_size", s)), A=20.0, alpha=1.0, f_max=1e7, f_min=-1e6,
                                omega=1.0, orthant_projection=orthant, number_of_iterations=n_it, return_best=True)
        orc = O.Oracle(pb)
        cpw = np.ones(pb.C)
        opt = O.OracleOptimizer(orc, od, m, np.zeros(pb.num_parameters), cpw, df=past,
                                df_geometry=pb.fixed_geometry() if past is not None else None)
        opt.run(n_it)
        best.append(float(opt.state.best_value))
        params = opt.best
        cp = np.ascontiguousarray(params.reshape(D, -1).T)
        past = orc.displacement_field(cp, cpw, past, pb.fixed_geometry() if past is not None else None)
        past = np.ascontiguousarray(past.reshape(ref.shape + (D,)))
        orc.close()
    return past, best
