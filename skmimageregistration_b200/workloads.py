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
