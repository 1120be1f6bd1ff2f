"""LCC where the reference's truncations sit on ties.

With the kernel support an exact multiple of the voxel spacing (9 mm = 6 voxels and 3 mm =
2 voxels at 1.5 mm) the window bounds trunc(inv*(p - o) - support/spacing + 1) are truncated from
exact integers, and with a neighbourhood stride above 1 a bound one voxel lower selects a
different neighbour lattice.  Windows with a single neighbour have LCC moments that are exactly
zero when every product is rounded on its own.  Both only come out as the reference's source
states them when the arithmetic is evaluated as written (GpuEvaluatorLCC.cu:94-191,
Kernel.h:158-171, ImageBase.h:51-59), so our path is held against the FP64 oracle and against the
reference's evaluator compiled with IEEE arithmetic (no fast math, no multiply-add contraction).
The reference's shipped -use_fast_math build contracts these expressions and is not asserted
against here: its own IEEE build differs from it by up to 1e-3 relative in value on these inputs.
"""
import os

import numpy as np
import pytest

from helpers import max_rel, rel_err
from oracle import oracle as O
from skmimageregistration_b200 import abi, synth
from skmimageregistration_b200 import register as R
from skmimageregistration_b200.evaluator import GpuKernelEvaluator, bspline_coefficients
from skmimageregistration_b200.problem import Problem

pytestmark = pytest.mark.gpu

SPACING = (1.5, 1.5, 1.5)
# (subsample, neighbourhood stride, sigma C4, sigma C0, control spacing): support = min(sigma)
CONFIGS = [(4, 6, 9.0, 18.0, 3.0), (2, 2, 3.0, 6.0, 1.5)]


def _images():
    fixed, moving, _ = synth.ct3d(seed=0, shape=(24, 32, 32))
    return R.threshold_rescale(fixed, (-1500, 3500)), R.threshold_rescale(moving, (-1500, 3500))


def _problem(kind, cfg, fixed, moving):
    sub, nbh, s4, s0, cps = cfg
    kw = {}
    if kind == "builder_tensors":             # the CT workload's combination: identity maxcov
        cov, tilt = R.anisotropic_tensor(fixed, SPACING, s4, 50.0, 2)
        kw = dict(weight_tensor=cov, maximum_weight=tilt if tilt >= 0 else 1.0,
                  maximum_eigenvalue_covariance=np.eye(3))
    elif kind == "random_tensors":            # maximum-eigenvalue covariance from the tensors
        a = np.random.default_rng(0).normal(size=fixed.shape + (3, 3)) * 0.25
        kw = dict(weight_tensor=np.einsum("...ij,...kj->...ik", a, a) + np.eye(3) * 0.9)
    return Problem(fixed=fixed, moving_coefficients=bspline_coefficients(moving), spacing=SPACING,
                   origin=(0.0,) * 3, sigma_c0=s0, sigma_c4=s4, cp_spacing=cps, subsample=sub,
                   subsample_neighborhood=nbh, **kw)


@pytest.mark.parametrize("cfg", CONFIGS, ids=["support6vox_stride6", "support2vox_stride2"])
@pytest.mark.parametrize("kind", ["stationary", "builder_tensors", "random_tensors"])
@pytest.mark.parametrize("alpha", [0.0, 0.3])
def test_lcc_on_ties_matches_oracle(cfg, kind, alpha):
    fixed, moving = _images()
    pb = _problem(kind, cfg, fixed, moving)
    cp = np.random.default_rng(1).normal(0, alpha, (pb.C, 3))
    cpw = np.ones(pb.C)
    ev = GpuKernelEvaluator(pb)
    orc = O.Oracle(pb)
    for call in range(2):                     # the second call redraws the sample shifts
        r, g = ev.getValueAndDerivative(abi.LCC, cp, cpw)
        ro, go = orc.evaluate(abi.LCC, cp, cpw)
        assert r["num_pixels_counted"] == ro["num_pixels_counted"]
        assert rel_err(r["measure"], ro["measure"]) <= 1e-5
        assert max_rel(g, go) <= 1e-4
    ev.close()
    orc.close()


@pytest.mark.skipif(not os.path.exists(O.ref_gpu_path(3, True, ieee=True)),
                    reason="reference evaluator (IEEE build) not built")
@pytest.mark.parametrize("cfg", CONFIGS[:1], ids=["support6vox_stride6"])
@pytest.mark.parametrize("kind", ["stationary", "builder_tensors", "random_tensors"])
def test_lcc_on_ties_matches_reference_ieee_build(cfg, kind):
    fixed, moving = _images()
    pb = _problem(kind, cfg, fixed, moving)
    cp = np.random.default_rng(1).normal(0, 0.3, (pb.C, 3))
    cpw = np.ones(pb.C)
    ev = GpuKernelEvaluator(pb)
    ref = O.RefGpu(pb, double=True, ieee=True)
    r, g = ev.getValueAndDerivative(abi.LCC, cp, cpw)
    rr, gr = ref.evaluate(abi.LCC, cp, cpw)
    assert r["num_pixels_counted"] == rr["num_pixels_counted"]
    assert rel_err(r["measure"], rr["measure"]) <= 1e-5
    assert max_rel(g, gr) <= 1e-4
    ev.close()
    ref.close()
