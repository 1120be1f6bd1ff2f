"""Device-memory inputs of the C-ABI (the multi-scale driver's device-resident path).

skm_evaluator_create reads the fixed image and the moving coefficients in place when they are
device memory, the frozen displacement field of a call may be device memory, and
skm_evaluate_displacement_field writes into device memory directly.  Results must equal those of
the host-array path bit for bit: the same conversions run on the device either way.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import make_problem
from skmimageregistration_b200 import abi
from skmimageregistration_b200.abi import Field
from skmimageregistration_b200.evaluator import GpuKernelEvaluator, check, lib

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

_dp = C.POINTER(C.c_double)


def _device_evaluator(pb, keep):
    """A GpuKernelEvaluator whose fixed image and coefficients the library reads from device memory."""
    fix = torch.tensor(np.ascontiguousarray(pb.fixed, np.float64), device="cuda")
    coe = torch.tensor(np.ascontiguousarray(pb.moving_coefficients, np.float64), device="cuda")
    keep += [fix, coe]
    ev = GpuKernelEvaluator.__new__(GpuKernelEvaluator)
    ev.problem = pb
    ev._desc = pb.desc()
    ev._desc.fixed_image = C.cast(fix.data_ptr(), _dp)
    ev._desc.moving_coefficients = C.cast(coe.data_ptr(), _dp)
    h = C.c_void_p()
    check(lib().skm_evaluator_create(C.byref(ev._desc), C.byref(h)))
    ev.h, ev.D, ev.C, ev._df_keep = h, pb.D, pb.C, None
    return ev


@pytest.mark.parametrize("D,kind,metric", [(3, "stationary", abi.NCC), (3, "weight_tensor", abi.MSE),
                                           (2, "weight_image", abi.NCC)])
def test_evaluator_from_device_images_matches_host(D, kind, metric):
    pb, cp, cpw = make_problem(D, kind, seed=123)
    keep = []
    ev_h = GpuKernelEvaluator(pb)
    ev_d = _device_evaluator(pb, keep)
    for e in (ev_h, ev_d):
        e.SetRegularizerRD(1e-2)
    r_h, g_h = ev_h.getValueAndDerivative(metric, cp, cpw)
    r_d, g_d = ev_d.getValueAndDerivative(metric, cp, cpw)
    assert r_h == r_d
    assert np.array_equal(g_h, g_d)
    ev_h.close()
    ev_d.close()


@pytest.mark.parametrize("D", [2, 3])
def test_device_field_in_and_out_matches_host(D):
    pb, cp, cpw = make_problem(D, "stationary", seed=124)
    ev = GpuKernelEvaluator(pb)
    rng = np.random.default_rng(5)
    df = np.ascontiguousarray(rng.normal(0, 0.5, (pb.n_texels, D)))
    host_out = ev.evaluateDisplacementField(cp, cpw, df)
    # the same call with the field and the destination in device memory
    df_dev = torch.tensor(df, device="cuda")
    out_dev = torch.zeros((pb.n_texels, D), dtype=torch.float64, device="cuda")
    f = Field()
    f.data = C.cast(df_dev.data_ptr(), _dp)
    f.geometry = pb.fixed_geometry()
    cp_aos = np.ascontiguousarray(cp, np.float64)
    w = np.ascontiguousarray(cpw, np.float64)
    check(lib().skm_evaluate_displacement_field(ev.h, cp_aos.ctypes.data_as(_dp), w.ctypes.data_as(_dp),
                                                C.byref(f), C.cast(out_dev.data_ptr(), _dp)))
    torch.cuda.synchronize()
    assert np.array_equal(out_dev.cpu().numpy(), host_out.reshape(pb.n_texels, D))
    ev.close()
