"""Small seeded registration problems shared by the tests."""
from __future__ import annotations

import numpy as np

from skmimageregistration_b200.problem import Problem


def smooth_volume(rng, shape, n_blobs=6):
    """Seeded smooth test image in [0, 1] (sum of Gaussian blobs + a ramp)."""
    grids = np.indices(shape, dtype=np.float64)
    img = 0.1 * grids[-1] / max(shape[-1], 1)
    for _ in range(n_blobs):
        c = [rng.uniform(0, n) for n in shape]
        s = rng.uniform(0.15, 0.35) * min(shape)
        r2 = sum((g - cc) ** 2 for g, cc in zip(grids, c))
        img = img + rng.uniform(0.3, 1.0) * np.exp(-r2 / (2 * s * s))
    img = (img - img.min()) / (img.max() - img.min())
    return img


def bspline_coefficients_host(image):
    """Coefficients via the FP64 oracle (test side only)."""
    from oracle import oracle as O
    return O.bspline_coefficients(image)


def make_problem(D=3, kind="stationary", subsample=1, nbh=1, shape=None, seed=0, sigma_c4=4.5, sigma_c0=9.0,
                 cp_spacing=2.0, spacing=None, origin=None, alpha_scale=1.0, weights=True, coeffs=None):
    """Returns (problem, cp (C,D) AoS, cpw (C,))."""
    rng = np.random.default_rng(seed)
    if shape is None:
        shape = (14, 16, 18) if D == 3 else (40, 44)
    spacing = spacing or tuple([1.0, 1.1, 0.9][:D])
    origin = origin or tuple([0.5, -1.0, 2.0][:D])
    fixed = smooth_volume(rng, shape)
    moving = smooth_volume(rng, shape)
    if coeffs is None:
        coeffs = bspline_coefficients_host(moving)
    kw = {}
    if kind == "weight_image":
        kw["weight_image"] = rng.uniform(0.6, 1.6, shape)
    elif kind == "weight_tensor":
        A = rng.normal(size=shape + (D, D)) * 0.25
        kw["weight_tensor"] = np.einsum("...ij,...kj->...ik", A, A) + np.eye(D) * 0.9
    pb = Problem(fixed=fixed, moving_coefficients=coeffs, spacing=spacing, origin=origin, sigma_c0=sigma_c0,
                 sigma_c4=sigma_c4, cp_spacing=cp_spacing, subsample=subsample, subsample_neighborhood=nbh, **kw)
    cp = rng.uniform(-1.0, 1.0, (pb.C, D)) * alpha_scale
    cpw = rng.uniform(0.5, 1.5, pb.C) if weights else np.ones(pb.C)
    return pb, cp, cpw


def rel_err(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


def max_rel(a, b):
    """max |a-b| relative to max |b| (norm-wise relative error of a field)."""
    a = np.asarray(a); b = np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def componentwise_rel(a, b, floor=1e-3):
    """Largest componentwise relative error |a_i - b_i| / |b_i| over the components whose
    reference magnitude |b_i| exceeds `floor` * max |b| (a small component can then not hide
    behind the largest one, as it can in the norm-wise max_rel)."""
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    sel = np.abs(b) > floor * np.max(np.abs(b))
    if not np.any(sel):
        return 0.0
    return float(np.max(np.abs(a[sel] - b[sel]) / np.abs(b[sel])))
