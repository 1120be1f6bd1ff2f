"""Named benchmark workloads (seeded synthetic inputs with the described shapes).

``ncc128``: 128x128x96 float volume pair (6 ellipsoids over a smooth background, sliding
shear + Wendland displacement), 1 mm voxels, control-point spacing 4 voxels
(32x32x24 = 24,576 points), kernel support 12 voxels (sigma_C4 = 12, sigma_C0 = 24, so
the transform and the "bilateral" RD regularizer share one kernel), NCC metric,
RD weight 1e-3, every voxel sampled (subsample 1).

``mse2d``: 256x256 blob image pair, control spacing 8 px, support 16 px, MSE, L1 1e-3.
"""
from __future__ import annotations

import numpy as np

from . import synth
from .abi import MetricDesc, OptimizerDesc
from .problem import Problem

WORKLOADS = {
    "ncc128": dict(shape=(96, 128, 128), spacing=(1.0, 1.0, 1.0), sigma_c4=12.0, sigma_c0=24.0, cp_spacing=4.0,
                   metric="ncc", rd=1e-3, l1=0.0, subsample=1),
    "mse2d": dict(shape=(256, 256), spacing=(1.0, 1.0), sigma_c4=16.0, sigma_c0=32.0, cp_spacing=8.0,
                  metric="mse", rd=0.0, l1=1e-3, subsample=1),
}


def make(name="ncc128", seed=0, coefficients=None):
    """Returns (problem, metric descriptor, optimizer descriptor, info dict).

    `coefficients(moving) -> padded B-spline coefficients`; defaults to the GPU prefilter.
    """
    w = WORKLOADS[name]
    if len(w["shape"]) == 3:
        fixed, moving, _ = synth.ellipsoids3d(seed=seed, shape=w["shape"])
    else:
        fixed, moving, _ = synth.blobs2d(seed=seed, shape=w["shape"])
    if coefficients is None:
        from .evaluator import bspline_coefficients as coefficients
    co = coefficients(moving)
    D = len(w["shape"])
    pb = Problem(fixed=fixed, moving_coefficients=co, spacing=w["spacing"], origin=(0.0,) * D,
                 sigma_c0=w["sigma_c0"], sigma_c4=w["sigma_c4"], cp_spacing=w["cp_spacing"],
                 subsample=w["subsample"], subsample_neighborhood=1)
    m = MetricDesc.make(w["metric"], rd=w["rd"], l1=w["l1"])
    o = OptimizerDesc.make(a=1.0, number_of_iterations=1 << 30,
                           orthant_projection=(w["l1"] > 0 and w["rd"] == 0))
    info = dict(workload=name, volume="x".join(str(s) for s in reversed(w["shape"])), control_points=pb.C,
                cp_grid="x".join(str(s) for s in pb.cp_size), support_voxels=min(w["sigma_c4"], w["sigma_c0"]),
                cp_spacing_voxels=w["cp_spacing"], metric=w["metric"], reg_rd=w["rd"], reg_l1=w["l1"],
                subsample=w["subsample"], seed=seed)
    return pb, m, o, info


def make_batch(n=64, seed=0, bases=4, lo=(64, 64, 64), hi=(160, 160, 128), coefficients=None):
    """Batched workload: `n` config-2-style pairs with sizes uniform in [lo, hi] (X, Y, Z voxels).

    Each pair is a crop (same box in both images, so the registration problem is intact) of one of
    `bases` seeded 160x160x128 ellipsoid pairs (6 ellipsoids over a smooth background + N(0, 0.02),
    sliding shear + Wendland displacement), rescaled to [0, 1]; control spacing 4 voxels, support
    12 voxels; even pairs NCC, odd pairs MSE, both with RD 1e-3.  Returns (problems, metric
    descriptors, optimizer descriptor, info dict)."""
    rng = np.random.default_rng(seed)
    base = [synth.ellipsoids3d(seed=seed * 1000 + k, shape=(hi[2], hi[1], hi[0]))[:2] for k in range(bases)]
    if coefficients is None:
        from .evaluator import bspline_coefficients as coefficients
    problems, metrics, sizes = [], [], []
    for i in range(n):
        size = [int(rng.integers(lo[d], hi[d] + 1)) for d in range(3)]        # X, Y, Z
        off = [int(rng.integers(0, hi[d] - size[d] + 1)) for d in range(3)]
        fixed, moving = base[int(rng.integers(0, bases))]
        sl = (slice(off[2], off[2] + size[2]), slice(off[1], off[1] + size[1]), slice(off[0], off[0] + size[0]))
        f = np.ascontiguousarray(fixed[sl])
        m = np.ascontiguousarray(moving[sl])
        pb = Problem(fixed=f, moving_coefficients=coefficients(m), spacing=(1.0, 1.0, 1.0), origin=(0.0, 0.0, 0.0),
                     sigma_c0=24.0, sigma_c4=12.0, cp_spacing=4.0, subsample=1, subsample_neighborhood=1)
        problems.append(pb)
        metrics.append(MetricDesc.make("ncc" if i % 2 == 0 else "mse", rd=1e-3))
        sizes.append(size)
    o = OptimizerDesc.make(a=1.0, number_of_iterations=1 << 30)
    texels = int(sum(np.prod(s) for s in sizes))
    info = dict(workload="batch%d" % n, pairs=n, sizes="uniform %dx%dx%d .. %dx%dx%d" % (tuple(lo) + tuple(hi)),
                total_voxels=texels, metrics="NCC (even pairs) / MSE (odd pairs), RD 1e-3",
                control_points=int(sum(pb.C for pb in problems)), cp_spacing_voxels=4.0, support_voxels=12.0,
                seed=seed)
    return problems, metrics, o, info
