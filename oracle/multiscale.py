"""FP64 restatements of the multi-scale driver and its preprocessing.

TEST INFRASTRUCTURE ONLY: imported by tests/ (and usable by bench.py's CPU leg), never by the
product.  Follows
  * GaussianSmoothing, include/itkUtils.h:139-150 (ITK DiscreteGaussianImageFilter: per-axis
    discrete Gaussian e^-t I_n(t), t = variance / spacing^2, grown until 1 - maximum_error of the
    mass, half width <= maximum_kernel_width, normalised; edge voxels repeated);
  * ThresholdImage + RescaleImage, include/itkUtils.h:45-110;
  * ComputeAnisotropicTensor, include/AnisotropicTensorUtils.h:37-371 (anisotropic_filtering false,
    as src/SKMReg.cxx:271 calls it): structure tensor, eigen system ordered by magnitude
    (include/itkSymmetricEigenDecompositionImageFilter.h, here numpy.linalg.eigh), direction
    weighting and covariance;
  * the scale loop of src/SKMReg.cxx:84-500 with the FP64 evaluator and optimizer of oracle.py,
    including the kernel weighting of :245-297.
ITK itself is not in this container: the ITK filters are restated from their published
algorithms (exact Bessel values, scipy.special.ive), so agreement with ITK is unpinned.
"""
from __future__ import annotations

import math

import numpy as np
from scipy.special import ive

from skmimageregistration_b200.abi import METRICS, MetricDesc, OptimizerDesc
from skmimageregistration_b200.problem import Problem, control_point_grid
from skmimageregistration_b200.register import current, full_config

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


def image_gradient(image, spacing):
    """itk::GradientImageFilter as ComputeAnisotropicTensor uses it (include/AnisotropicTensorUtils.h:65-68):
    per axis (f[i+1] - f[i-1]) / (2 spacing), an edge texel's missing neighbour replaced by the
    texel itself (zero-flux Neumann).  Returns (..., D), component 0 = x."""
    f = np.asarray(image, np.float64)
    D = f.ndim
    g = np.empty(f.shape + (D,))
    for d in range(D):
        ax = D - 1 - d
        n = f.shape[ax]
        idx = np.arange(n)
        hi = np.take(f, np.minimum(idx + 1, n - 1), axis=ax)
        lo = np.take(f, np.maximum(idx - 1, 0), axis=ax)
        g[..., d] = (hi - lo) / (2.0 * float(spacing[d]))
    return g


def structure_tensor(image, spacing, sigma, weight):
    """K_{sigma/4} * (grad u_sigma grad u_sigma^T) of weight * image (AnisotropicTensorUtils.h:54-155):
    smoothing with variance sigma, gradient, outer product, every component smoothed with variance
    sigma / 4.  Returns (..., D, D)."""
    f = np.asarray(image, np.float64) * float(weight)
    D = f.ndim
    g = image_gradient(gaussian_smooth(f, spacing, float(sigma)), spacing)
    T = np.empty(f.shape + (D, D))
    for i in range(D):
        for j in range(i, D):
            T[..., i, j] = gaussian_smooth(g[..., i] * g[..., j], spacing, float(sigma) / 4.0)
            T[..., j, i] = T[..., i, j]
    return T


def covariance_from_structure(T, alignment_direction=2):
    """The per-texel steps of ComputeAnisotropicTensor after the structure tensor
    (AnisotropicTensorUtils.h:160-371), on (..., D, D) structure tensors.

    Eigen decomposition ordered by magnitude, rows = eigenvalue * eigenvector
    (include/itkSymmetricEigenDecompositionImageFilter.h); where every row is longer than 1e-8 the
    main (largest) row is weighted by (|n x e_align| + 1e-10)^2 / sqrt(D) (only for an alignment
    axis < D), p = |main row|^1.5, the main direction gets length 1/(1+p), the others
    1 + p/(1+p), else the identity; then the rows are flipped and transposed and the covariance is
    U diag(column norms) U^T (:316-360).  Returns (covariance (..., D, D), maximum tilt = the largest
    |main row| over the texels that passed, -DBL_MAX when none did, number of non-positive
    determinants)."""
    T = np.asarray(T, np.float64)
    D = T.shape[-1]
    shape = T.shape[:-2]
    flat = T.reshape(-1, D, D)
    lam, vec = np.linalg.eigh(flat)                        # columns of vec are eigenvectors
    order = np.argsort(np.abs(lam), axis=1, kind="stable")
    lam = np.take_along_axis(lam, order, 1)
    vec = np.take_along_axis(vec, order[:, None, :], 2)
    rows = vec.transpose(0, 2, 1) * lam[:, :, None]        # row k = lam_k v_k, |lam| ascending
    mag = np.linalg.norm(rows, axis=2)
    ok = np.all(mag > 1e-8, axis=1)
    safe = np.where(mag > 0, mag, 1.0)
    normalized = rows[:, D - 1, :] / safe[:, D - 1:D]
    main = rows[:, D - 1, :].copy()
    if 0 <= alignment_direction < D:
        md = np.zeros(D)
        md[alignment_direction] = 1.0
        if D == 2:
            cross = np.abs(normalized[:, 0] * md[1] - normalized[:, 1] * md[0])
        else:
            cross = np.linalg.norm(np.cross(normalized, md), axis=1)
        factor = (cross + 1e-10) ** 2 / math.sqrt(D)
        main = main * factor[:, None]
    rev = np.linalg.norm(main, axis=1)
    p = rev ** 1.5
    new = np.empty_like(rows)
    new[:, D - 1, :] = normalized / (1.0 + p)[:, None]
    for k in range(D - 1):
        new[:, k, :] = rows[:, k, :] / safe[:, k:k + 1] * (1.0 + p / (1.0 + p))[:, None]
    M = new[:, ::-1, :].transpose(0, 2, 1)                 # flipud().transpose(): column 0 = main
    M = np.where(ok[:, None, None], M, np.eye(D)[None])
    max_tilt = float(rev[ok].max()) if ok.any() else -np.finfo(np.float64).max
    s = np.linalg.norm(M, axis=1)                          # column norms
    U = M / np.where(s > 0, s, 1.0)[:, None, :]
    cov = np.einsum("nik,nk,njk->nij", U, s, U)
    cov = np.where((s[:, 0] < 1e-8)[:, None, None], np.eye(D)[None], cov)
    bad = int(np.count_nonzero(~(np.linalg.det(cov) > 0)))
    return cov.reshape(shape + (D, D)), max_tilt, bad


def anisotropic_tensor(image, spacing, sigma, weight, alignment_direction=2):
    """ComputeAnisotropicTensor (include/AnisotropicTensorUtils.h:37-371) with anisotropic_filtering
    false, as src/SKMReg.cxx:271 and :284 call it: (covariance (..., D, D), maximum tilt)."""
    cov, tilt, bad = covariance_from_structure(structure_tensor(image, spacing, sigma, weight), alignment_direction)
    if bad:
        raise ValueError("covariance tensor not positive definite at %d texels" % bad)
    return cov, tilt


def level_weighting(tar_s, spacing, c, s, guidance_image=None, weight_tensor=None, weight_image=None):
    """Problem keyword arguments for the kernel weighting of level s (src/SKMReg.cxx:245-297 with
    SetWeightingImage / SetWeightingTensor, include/itkTransformAdapter.hxx:312-365)."""
    D = np.asarray(tar_s).ndim
    tw = float(current(c, "tensor_weights", s))
    tensor, weight, cov = None, None, None
    if tw > 0:
        src = tar_s if guidance_image is None else np.asarray(guidance_image, np.float64)
        tensor, tilt = anisotropic_tensor(src, spacing, float(np.float32(current(c, "sigma_C4", s))), tw, 2)
        weight, cov = (tilt, np.eye(D)) if tilt >= 0 else (1.0, np.eye(D))
    elif tw == 0 and weight_tensor is not None:
        tensor = np.asarray(weight_tensor, np.float64)
        flat = tensor.reshape(-1, D, D)
        if np.any(~(np.linalg.det(flat) > 0)):
            raise ValueError("weighting tensors must be positive definite")
        ev = np.abs(np.linalg.eigvalsh(flat)[:, -1])
        k = int(np.argmax(ev))
        weight, cov = float(ev[k]), flat[k].copy()
    if weight_image is not None:
        wi = np.asarray(weight_image, np.float64)
        return dict(weight_image=wi, maximum_weight=weight if tensor is not None else float(wi.max()))
    if tensor is not None:
        return dict(weight_tensor=tensor, maximum_weight=weight, maximum_eigenvalue_covariance=cov)
    return {}


def _mirror(k, n):
    period = 2 * (n - 1)
    if period <= 0:
        return np.zeros_like(k)
    k = np.mod(k, period)
    return np.where(k < n, k, period - k)


def warp_image(image, displacement, image_spacing, image_origin, field_spacing, field_origin, order=3,
               default_value=0.0):
    """I(p + u(p)) on the field's grid (WarpImage, include/itkUtils.h:163-178, order 3; the final
    resampling of src/SKMReg.cxx:504-522, order 1).  Outside [-0.5, size - 0.5) in continuous index:
    default_value.  Order 1: multilinear with clamped neighbours; order 3: cubic B-spline of the
    evaluator's prefiltered coefficients at floor(x) - 1 .. floor(x) + 2, whole-sample mirrored."""
    img = np.asarray(image, np.float64)
    u = np.asarray(displacement, np.float64)
    D = img.ndim
    isize = tuple(reversed(img.shape))
    fgrid = u.shape[:-1]
    idx = np.indices(fgrid, dtype=np.float64)             # numpy order: axis 0 = z (or y)
    ci, inside = [], np.ones(fgrid, bool)
    for d in range(D):
        p = field_origin[d] + field_spacing[d] * idx[D - 1 - d] + u[..., d]
        c = (p - image_origin[d]) / image_spacing[d]
        inside &= (c >= -0.5) & (c < isize[d] - 0.5)
        ci.append(c)
    if order == 3:
        coef = O.bspline_coefficients(img)[tuple(slice(1, n + 1) for n in img.shape)]
    else:
        coef = img
    taps = 2 if order == 1 else 4
    W, I = [], []
    for d in range(D):
        b = np.floor(ci[d])
        t = ci[d] - b
        b = b.astype(np.int64)
        if order == 1:
            W.append([1.0 - t, t])
            I.append([np.clip(b, 0, isize[d] - 1), np.clip(b + 1, 0, isize[d] - 1)])
        else:
            s = 1.0 - t
            W.append([s ** 3 / 6.0, 2.0 / 3.0 - t * t + 0.5 * t ** 3, 2.0 / 3.0 - s * s + 0.5 * s ** 3, t ** 3 / 6.0])
            I.append([_mirror(b - 1 + k, isize[d]) for k in range(4)])
    out = np.zeros(fgrid)
    for corner in np.ndindex(*([taps] * D)):
        w = np.ones(fgrid)
        for d in range(D):
            w = w * W[d][corner[d]]
        sel = tuple(I[d][corner[d]] for d in reversed(range(D)))
        out += w * coef[sel]
    return np.where(inside, out, default_value)


def jacobian_determinant(field, spacing):
    """JacobianDeterminant (include/itkUtils.h:153-161): det(I + du/dx), central differences over
    2 spacing with edge texels repeated."""
    u = np.asarray(field, np.float64)
    D = u.shape[-1]
    J = np.zeros(u.shape[:-1] + (D, D))
    for j in range(D):
        ax = D - 1 - j
        n = u.shape[ax]
        k = np.arange(n)
        hi = np.take(u, np.minimum(k + 1, n - 1), axis=ax)
        lo = np.take(u, np.maximum(k - 1, 0), axis=ax)
        J[..., :, j] = (hi - lo) / (2.0 * float(spacing[j]))
    J += np.eye(D)
    return np.linalg.det(J)


def register(reference, target, spacing, origin, config, guidance_image=None, weight_tensor=None, weight_image=None,
             initial_displacement=None):
    """The scale loop with the FP64 evaluator / optimizer; returns (displacement, per-level best values)."""
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
    first = 0
    ra = int(c.get("restart_at", 0))
    if 1 < ra <= int(c["num_scales"]) and initial_displacement is not None:
        first = ra - 1
        past = np.ascontiguousarray(np.asarray(initial_displacement, np.float64))
    for s in range(first, int(c["num_scales"])):
        var = float(current(c, "smoothing_variance", s))
        ref_s = gaussian_smooth(ref, spacing, var) if var > 1e-5 else ref
        tar_s = gaussian_smooth(tar, spacing, var) if var > 1e-5 else tar
        s4, s0 = float(current(c, "sigma_C4", s)), float(current(c, "sigma_C0", s))
        smin = np.float32(min(np.float32(s4), np.float32(s0)))
        scaler = float(c["cp_spacing_scaler"])
        cps = float(smin / np.float32(1.0)) if scaler < 1 else float(smin / np.float32(scaler))
        pb = Problem(fixed=tar_s, moving_coefficients=O.bspline_coefficients(ref_s), spacing=spacing, origin=origin,
                     sigma_c0=s0, sigma_c4=s4, cp_spacing=cps, subsample=int(current(c, "sampling_rate", s)),
                     subsample_neighborhood=int(current(c, "neighborhood_sampling", s)),
                     **level_weighting(tar_s, spacing, c, s, guidance_image, weight_tensor, weight_image))
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
