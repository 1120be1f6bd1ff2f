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
    txt = open(os.path.join(ROOT, "include", "skm_gpu.h")).read()
    return sorted(set(re.findall(r"\b(skm_[a-z0-9_]+)\s*\(", txt)))


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
    assert lib.skm_abi_version() == 4


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
