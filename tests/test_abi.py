"""The C-ABI library without a GPU: it loads, exports every declared symbol, and
rejects invalid arguments with the reference's validation rules (no compute calls)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from helpers import make_problem
from skmimageregistration_b200 import abi, build
from skmimageregistration_b200 import evaluator as E

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    """Every entry point declared by the C headers (include/skm_gpu.h, include/skm_warmstart.h)."""
    names = set()
    for h in ("skm_gpu.h", "skm_warmstart.h"):
        txt = open(os.path.join(ROOT, "include", h)).read()
        names |= set(re.findall(r"\b(skm_[a-z0-9_]+)\s*\(", txt))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    build.build()
    return E.lib()


def test_library_exports_every_declared_symbol(lib):
    names = declared_symbols()
    assert len(names) >= 17
    for n in names:
        assert hasattr(lib, n), n


def test_abi_version(lib):
    assert lib.skm_abi_version() == 7


def _create(pb):
    d = pb.desc()
    h = C.c_void_p()
    rc = E.lib().skm_evaluator_create(C.byref(d), C.byref(h))
    return rc, E.lib().skm_last_error().decode()


@pytest.mark.parametrize("mutate,msg", [
    (lambda d: setattr(d, "subsample", 0), "subsample"),
    (lambda d: setattr(d, "subsample", 101), "subsample"),
    (lambda d: setattr(d, "subsample_neighborhood", 0), "neighborhood"),
    (lambda d: setattr(d, "sigma_c0", 0.0), "positive"),
    (lambda d: setattr(d, "sigma_c4", -1.0), "positive"),
    (lambda d: setattr(d, "dimensions", 4), "dimensions"),
    (lambda d: setattr(d, "num_parameters", 5), "num_parameters"),
])
def test_invalid_descriptor_rejected(lib, mutate, msg):
    pb, _, _ = make_problem(3, shape=(6, 7, 8))
    d = pb.desc()
    mutate(d)
    h = C.c_void_p()
    rc = lib.skm_evaluator_create(C.byref(d), C.byref(h))
    assert rc == abi.SKM_ERR_INVALID
    assert msg in lib.skm_last_error().decode()


def test_nonpositive_weight_image_rejected(lib):
    pb, _, _ = make_problem(3, "weight_image", shape=(6, 7, 8))
    pb.weight_image[1, 2, 3] = 0.0                  # itkTransformAdapter.hxx:325-327
    rc, msg = _create(pb)
    assert rc == abi.SKM_ERR_INVALID and "strictly positive" in msg


def test_indefinite_tensor_rejected(lib):
    pb, _, _ = make_problem(3, "weight_tensor", shape=(6, 7, 8))
    pb.weight_tensor[0, 0, 0] = -np.eye(3)          # itkTransformAdapter.hxx:346-350
    rc, msg = _create(pb)
    assert rc == abi.SKM_ERR_INVALID and "positive definite" in msg


def test_null_arguments(lib):
    assert lib.skm_evaluator_create(None, None) == abi.SKM_ERR_INVALID
    assert lib.skm_get_value(None, 0, None, None, None, 1, None) == abi.SKM_ERR_STATE
    assert lib.skm_optimizer_run(None, 1) == abi.SKM_ERR_STATE


def test_no_cpu_fallback_without_device(lib):
    """Without a CUDA device a valid descriptor fails loudly instead of computing on the host."""
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    pb, _, _ = make_problem(3, shape=(6, 7, 8))
    rc, msg = _create(pb)
    assert rc == abi.SKM_ERR_CUDA
    assert "no CPU fallback" in msg


@pytest.mark.parametrize("which", ["control_points", "fixed_image", "result"])
def test_noalloc_rejects_misaligned_buffers_before_launching(lib, which):
    """skm_value_noalloc reads control points as float4: a buffer that is not 16-byte aligned
    (and images / result not aligned to their element type) is rejected with SKM_ERR_INVALID
    before any CUDA call, so this runs without a GPU."""
    fp, dp = C.POINTER(C.c_float), C.POINTER(C.c_double)
    lib.skm_value_noalloc.argtypes = [C.c_int32, C.c_int32, C.POINTER(abi.Geometry), fp, C.POINTER(abi.Geometry), fp,
                                      C.POINTER(abi.Geometry), fp, C.c_double, C.c_double, dp, C.c_void_p]
    lib.skm_value_noalloc.restype = C.c_int
    buf = (C.c_double * 64)()                       # 8-byte aligned host storage standing in for device buffers
    base = C.addressof(buf)
    base += (-base) % 16                            # 16-byte aligned start
    ptrs = dict(control_points=base, fixed_image=base, result=base)
    ptrs[which] = base + {"control_points": 4, "fixed_image": 2, "result": 4}[which]
    g = abi.Geometry.make([4, 4, 4])
    rc = lib.skm_value_noalloc(3, abi.NCC, C.byref(g), C.cast(ptrs["fixed_image"], fp), C.byref(g),
                               C.cast(base, fp), C.byref(g), C.cast(ptrs["control_points"], fp), 8.0, 4.0,
                               C.cast(ptrs["result"], dp), None)
    assert rc == abi.SKM_ERR_INVALID
    assert "aligned" in lib.skm_last_error().decode()
