"""Generate the golden fixtures of tests/golden/ from the reference itself.

Run from the repository root after `make -C oracle ref` has compiled the reference's
own host/device math headers from the reference checkout into oracle/_ref/:

    python tests/golden/make_golden.py

It writes reference_host_kat.npz: cubic B-spline prefilter coefficients, B-spline
values/gradients with inside flags, GKernel<float> values for the three kernel kinds,
maxEigenValue results and the UniformRng grid-shift stream -- every number computed by
the reference's own code on seeded inputs.  The oracle is checked against this file in
tests/test_oracle_golden.py.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from skmimageregistration_b200.abi import Geometry  # noqa: E402
from skmimageregistration_b200.problem import Problem  # noqa: E402

dp = C.POINTER(C.c_double)
ip = C.POINTER(C.c_int32)


def main():
    out = {}
    rng = np.random.default_rng(20161)
    for D in (2, 3):
        R = O.ref_host(D)
        if R is None:
            raise SystemExit("oracle/_ref not built: run `make -C oracle ref`")
        shape = (9, 10, 11) if D == 3 else (13, 17)
        img = rng.uniform(0, 1, shape)
        size = (C.c_int32 * 3)(*(list(reversed(shape)) + [1] * (3 - D)))
        co = np.zeros(tuple(s + 3 for s in shape))
        R.skmref_bspline_coefficients(size, img.ctypes.data_as(dp), co.ctypes.data_as(dp))
        out["bs%d_image" % D] = img
        out["bs%d_coeffs" % D] = co
        g = Geometry.make(list(reversed(shape)), [0.25] * D, [1.2] * D)
        pts = rng.uniform(-2.0, 14.0, (600, D))
        pts[:20] = np.round(pts[:20])                   # exact lattice points
        pts[20:40, 0] = -0.5 * 1.2 + 0.25 + rng.uniform(-1e-9, 1e-9, 20)   # the inside boundary
        ins = np.zeros(600, np.int32)
        val = np.zeros(600)
        grd = np.zeros((600, D))
        R.skmref_bspline_sample(co.ctypes.data_as(dp), C.byref(g), 600, pts.ctypes.data_as(dp),
                                ins.ctypes.data_as(ip), val.ctypes.data_as(dp), grd.ctypes.data_as(dp))
        out["bs%d_geom" % D] = np.array([0.25, 1.2])
        out["bs%d_points" % D] = pts
        out["bs%d_inside" % D] = ins
        out["bs%d_values" % D] = val
        out["bs%d_grads" % D] = grd

        kshape = (12, 13, 14) if D == 3 else (21, 23)
        for kind in ("stationary", "weight_image", "weight_tensor"):
            kw = {}
            if kind == "weight_image":
                kw["weight_image"] = rng.uniform(0.5, 2.0, kshape)
            if kind == "weight_tensor":
                A = rng.normal(size=kshape + (D, D)) * 0.3
                kw["weight_tensor"] = np.einsum("...ij,...kj->...ik", A, A) + np.eye(D) * 0.8
            pb = Problem(rng.uniform(0, 1, kshape), np.zeros(tuple(s + 3 for s in kshape)), (1.0,) * D,
                         (0.0,) * D, sigma_c0=8.0, sigma_c4=5.0, cp_spacing=2.0, **kw)
            d = pb.desc()
            p = rng.uniform(0.5, 10.5, (800, D))
            q = p + rng.normal(0, 3.0, (800, D))
            q = np.clip(q, 0.0, 10.9)
            k = np.zeros(800)
            R.skmref_kernel_values(C.byref(d), 800, p.ctypes.data_as(dp), q.ctypes.data_as(dp),
                                   k.ctypes.data_as(dp))
            key = "k%d_%s" % (D, kind)
            out[key + "_p"] = p
            out[key + "_q"] = q
            out[key + "_k"] = k
            for name in ("weight_image", "weight_tensor"):
                if name in kw:
                    out[key + "_" + name] = kw[name]
        mats = []
        eig = []
        for _ in range(200):
            A = rng.normal(size=(D, D))
            M = A @ A.T + 0.1 * np.eye(D)
            if len(mats) < 10:
                M = np.diag(np.diag(M))                 # diagonal branch (triSq == 0)
            mats.append(M)
            eig.append(R.skmref_max_eigenvalue(np.ascontiguousarray(M).ctypes.data_as(dp)))
        out["eig%d_m" % D] = np.array(mats)
        out["eig%d_v" % D] = np.array(eig)
        n = 5000
        sh = np.zeros((n, D), np.int32)
        R.skmref_grid_shifts(n, 4, sh.ctypes.data_as(ip))
        out["shifts%d_sub4" % D] = sh
    stream = np.zeros(64, np.uint32)
    O.ref_host(3).skmref_rng_stream(64, stream.ctypes.data_as(C.POINTER(C.c_uint32)))
    out["rng_stream"] = stream
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_host_kat.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
