"""The oracle on the LCC tie configuration that tests/test_lcc_ties_gpu.py runs on the GPU.

Support 9 mm at 1.5 mm spacing (6 voxels), subsample 4, neighbourhood stride 6: every window's
lower bound is truncated from an exact integer, and some windows hold a single neighbour (their
LCC moments are exactly zero when rounded as written, GpuEvaluatorLCC.cu:180-190).  The oracle must
treat the stationary kernel and identity tensors with an identity maximum-eigenvalue covariance
(support 9 / sqrt(2 / maxEig(I + I)) = 9, Kernel.h:158-171) identically, to the last bit.
"""
import numpy as np

from oracle import oracle as O
from skmimageregistration_b200 import synth
from skmimageregistration_b200.problem import Problem

SHAPE = (24, 32, 32)
SP = 1.5


def _problem(**kw):
    fixed, moving, _ = synth.ct3d(seed=0, shape=SHAPE)
    return Problem(fixed=fixed, moving_coefficients=O.bspline_coefficients(moving), spacing=(SP,) * 3,
                   origin=(0.0,) * 3, sigma_c0=18.0, sigma_c4=9.0, cp_spacing=3.0, subsample=4,
                   subsample_neighborhood=6, **kw)


def test_configuration_has_integer_bounds_and_single_neighbour_windows():
    Z, Y, X = SHAPE
    n = np.array([X, Y, Z])
    ss = n // 4
    shifts, _ = O.pcg32_shifts(int(np.prod(ss)), 3, 4)
    half = 9.0 / SP
    assert half == int(half)                                  # support on the voxel lattice
    single = 0
    for t, s in enumerate(shifts):
        c = np.array([t % ss[0], (t // ss[0]) % ss[1], t // (ss[0] * ss[1])])
        p = c * 4 + s
        assert np.all((1.0 / SP) * (SP * p) == p)             # local coordinates land on integers
        lo = np.clip((p - half + 1.0).astype(int), 0, n - 1)
        hi = np.clip((p + half).astype(int), 0, n - 1)
        count = 0
        for z in range(lo[2], hi[2] + 1, 6):
            for y in range(lo[1], hi[1] + 1, 6):
                for x in range(lo[0], hi[0] + 1, 6):
                    r = np.sqrt(np.sum(((p - np.array([x, y, z])) * SP) ** 2)) / 9.0
                    count += (1.0 - r ** 10) > 0.0
        single += count == 1
    assert single > 0


def test_oracle_stationary_equals_identity_tensors_on_ties():
    eye = np.broadcast_to(np.eye(3), SHAPE + (3, 3)).copy()
    a = _problem()
    b = _problem(weight_tensor=eye, maximum_weight=1.0, maximum_eigenvalue_covariance=np.eye(3))
    cp, cpw = np.zeros((a.C, 3)), np.ones(a.C)
    oa, ob = O.Oracle(a), O.Oracle(b)
    ra, ga = oa.evaluate(2, cp, cpw)
    rb, gb = ob.evaluate(2, cp, cpw)
    oa.close()
    ob.close()
    assert ra["num_pixels_counted"] == rb["num_pixels_counted"]
    assert ra["measure"] == rb["measure"]
    assert np.array_equal(ga, gb)
