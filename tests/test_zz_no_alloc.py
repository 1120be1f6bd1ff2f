"""skm_value_noalloc: the metric value for callers that cannot allocate device memory.

Such callers (a framework that owns the device memory budget, a real-time loop that
must avoid cudaMalloc's implicit synchronisation) hand in device buffers for every input
and for the result; the entry point itself allocates nothing and keeps its partial sums
in a fixed array inside the library.  This file checks it through the C-ABI against
the allocating entry point skm_get_value on two calls in a row (the second call reuses
the array the first one left behind), within the value tolerance of the parity tests.
It is collected last so that a failure here cannot stop the rest of the suite.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import make_problem, rel_err
from skmimageregistration_b200 import abi
from skmimageregistration_b200.evaluator import GpuKernelEvaluator, lib

pytestmark = pytest.mark.gpu

TOL_VALUE = 1e-5

_fp = C.POINTER(C.c_float)
_dp = C.POINTER(C.c_double)


def _bind():
    L = lib()
    L.skm_value_noalloc.argtypes = [C.c_int32, C.c_int32, C.POINTER(abi.Geometry), _fp, C.POINTER(abi.Geometry), _fp,
                                    C.POINTER(abi.Geometry), _fp, C.c_double, C.c_double, _dp, C.c_void_p]
    L.skm_value_noalloc.restype = C.c_int
    return L


def _noalloc_value(L, torch, pb, metric, cp, cpw, stream):
    """Device inputs prepared by the caller; the call itself allocates nothing."""
    dev = torch.device("cuda")
    fixed = torch.tensor(pb.fixed.astype(np.float32), device=dev).contiguous()
    coeffs = torch.tensor(pb.moving_coefficients.astype(np.float32), device=dev).contiguous()
    rec = np.zeros((pb.C, 4), np.float32)
    rec[:, :pb.D] = cp
    rec[:, 3] = cpw
    cps = torch.tensor(rec, device=dev).contiguous()
    out = torch.full((2,), float("nan"), dtype=torch.float64, device=dev)
    fg, mg, cg = pb.fixed_geometry(), pb.moving_geometry(), pb.cp_geometry()
    torch.cuda.synchronize()
    rc = L.skm_value_noalloc(pb.D, metric, C.byref(fg), C.cast(fixed.data_ptr(), _fp), C.byref(mg),
                             C.cast(coeffs.data_ptr(), _fp), C.byref(cg), C.cast(cps.data_ptr(), _fp),
                             pb.sigma_c0, pb.sigma_c4, C.cast(out.data_ptr(), _dp), C.c_void_p(stream))
    assert rc == 0, L.skm_last_error().decode()
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("D", [2, 3])
@pytest.mark.parametrize("metric", [abi.MSE, abi.NCC])
def test_noalloc_value_matches_allocating_entry_point(D, metric):
    torch = pytest.importorskip("torch")
    L = _bind()
    pb, cp, cpw = make_problem(D, seed=81)
    ev = GpuKernelEvaluator(pb)
    stream = torch.cuda.current_stream().cuda_stream
    for scale in (1.0, 0.5):                      # two calls in a row, different parameters
        got = _noalloc_value(L, torch, pb, metric, cp * scale, cpw, stream)
        ref = ev.getValue(metric, cp * scale, cpw)
        assert int(got[1]) == ref["num_pixels_counted"]
        assert rel_err(got[0], ref["measure"]) <= TOL_VALUE, (got, ref)


def test_noalloc_rejects_images_beyond_its_limit():
    pytest.importorskip("torch")
    L = _bind()
    D = 3
    big = abi.Geometry.make([256, 128, 65])       # 2,129,920 texels > 2,097,152
    dummy = (C.c_float * 4)()
    res = (C.c_double * 2)()
    rc = L.skm_value_noalloc(D, abi.NCC, C.byref(big), dummy, C.byref(big), dummy, C.byref(abi.Geometry.make([4, 4, 4])),
                             dummy, 8.0, 4.0, res, None)
    assert rc == abi.SKM_ERR_INVALID
    assert "at most 2097152" in L.skm_last_error().decode()
