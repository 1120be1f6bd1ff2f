"""The FP64 oracle against numbers computed by the reference's own code.

tests/golden/reference_host_kat.npz holds outputs of the reference's host-compiled
math headers (include/cuda/{BsplineImage,Kernel,Mat,UniformRng}.h), produced by
tests/golden/make_golden.py.  Integer results (inside flags, grid shifts, RNG) must
match exactly; double-precision B-spline results to round-off; kernel values to the
reference's float precision (GKernel<float>, Kernel.h:209).
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from skmimageregistration_b200.abi import Geometry
from skmimageregistration_b200.problem import Problem

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_host_kat.npz"))


@pytest.mark.parametrize("D", [2, 3])
def test_bspline_prefilter_matches_reference(D):
    co = O.bspline_coefficients(G["bs%d_image" % D])
    ref = G["bs%d_coeffs" % D]
    np.testing.assert_allclose(co, ref, rtol=0, atol=1e-12 * np.abs(ref).max())


@pytest.mark.parametrize("D", [2, 3])
def test_bspline_sampling_matches_reference(D):
    co = G["bs%d_coeffs" % D]
    o, s = G["bs%d_geom" % D]
    shape = G["bs%d_image" % D].shape
    g = Geometry.make(list(reversed(shape)), [o] * D, [s] * D)
    ins, val, grd = O.bspline_sample(co, g, G["bs%d_points" % D])
    np.testing.assert_array_equal(ins, G["bs%d_inside" % D])
    np.testing.assert_allclose(val, G["bs%d_values" % D], rtol=0, atol=1e-12)
    np.testing.assert_allclose(grd, G["bs%d_grads" % D], rtol=0, atol=1e-12)


@pytest.mark.parametrize("D", [2, 3])
@pytest.mark.parametrize("kind", ["stationary", "weight_image", "weight_tensor"])
def test_kernel_values_match_reference(D, kind):
    key = "k%d_%s" % (D, kind)
    kshape = (12, 13, 14) if D == 3 else (21, 23)
    kw = {}
    for name in ("weight_image", "weight_tensor"):
        if key + "_" + name in G:
            kw[name] = G[key + "_" + name]
    pb = Problem(np.zeros(kshape), np.zeros(tuple(s + 3 for s in kshape)), (1.0,) * D, (0.0,) * D,
                 sigma_c0=8.0, sigma_c4=5.0, cp_spacing=2.0, **kw)
    k = O.kernel_values(pb.desc(), G[key + "_p"], G[key + "_q"])
    ref = G[key + "_k"]
    assert np.isfinite(ref).all()
    # reference kernel is float (GKernel<float>): agreement to float round-off
    np.testing.assert_allclose(k, ref, rtol=0, atol=2e-6)
    assert (k > 0).sum() > 100


@pytest.mark.parametrize("D", [2, 3])
def test_grid_shifts_match_reference(D):
    sh, _ = O.pcg32_shifts(5000, D, 4)
    np.testing.assert_array_equal(sh, G["shifts%d_sub4" % D])


def test_rng_stream_matches_reference():
    import ctypes as C
    st = C.c_uint64(0xBA5EBA11DEADBEEF)
    got = [O.lib().ora_pcg32_next(C.byref(st)) for _ in range(64)]
    np.testing.assert_array_equal(np.array(got, np.uint32), G["rng_stream"])
