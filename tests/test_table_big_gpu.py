"""The phase-table path at coarse scale levels: control spacing 8 and 16 voxels (512 and 4096 phases),
where the tables no longer fit in shared memory and the large-phase kernels run (tables in global
memory / L2).  Compared with the FP64 oracle and with the generic kernels: values 1e-5 relative,
derivatives 1e-4 of the largest component, pixel counts exact; and the multi-scale driver's coarse
levels take this path."""
import numpy as np
import pytest

from helpers import make_problem, max_rel, rel_err
from oracle import oracle as O
from skmimageregistration_b200 import abi
from skmimageregistration_b200.evaluator import GpuKernelEvaluator

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("h,shape,s4", [(8, (30, 34, 38), 24.0), (16, (40, 44, 48), 48.0), (16, (66, 70), 48.0)])
@pytest.mark.parametrize("metric", [abi.MSE, abi.NCC])
def test_large_phase_table_matches_oracle_and_generic(h, shape, s4, metric):
    D = len(shape)
    pb, cp, cpw = make_problem(D, "stationary", shape=shape, seed=300 + h, sigma_c4=s4, sigma_c0=2 * s4,
                               cp_spacing=float(h), spacing=(1.0,) * D, origin=tuple([0.5, -1.0, 2.0][:D]),
                               alpha_scale=3.0)
    ev = GpuKernelEvaluator(pb)
    # 3-D: 512 / 4096 phases, the large-phase kernels; 2-D h = 16: 256 phases of one (px, py) row per
    # block, the shared-memory-table kernels (too many phases for the tensor-core GEMMs either way)
    assert ev.path() == GpuKernelEvaluator.TABLE, ev.describe()
    assert ev.describe()["table_phases"] == h ** D
    ev.SetRegularizerRD(1e-2)
    r, g = ev.getValueAndDerivative(metric, cp, cpw)
    orc = O.Oracle(pb)
    orc.set_regularizers(rd=1e-2)
    ro, go = orc.evaluate(metric, cp, cpw)
    assert r["num_pixels_counted"] == ro["num_pixels_counted"]
    assert rel_err(r["measure"], ro["measure"]) <= 1e-5
    assert rel_err(r["reg_value_rd"], ro["reg_value_rd"]) <= 1e-5
    assert max_rel(g, go) <= 1e-4
    u = ev.evaluateDisplacementField(cp, cpw)
    assert max_rel(u, orc.displacement_field(cp, cpw)) <= 1e-5
    assert ev.path(GpuKernelEvaluator.REQ_GENERIC) == GpuKernelEvaluator.GENERIC
    r2, g2 = ev.getValueAndDerivative(metric, cp, cpw)
    assert rel_err(r["measure"], r2["measure"]) <= 1e-5
    assert max_rel(g, g2) <= 1e-4
