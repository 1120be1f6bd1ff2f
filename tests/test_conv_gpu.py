"""The warm start's tcgen05 convolution kernels (csrc/skm_conv.cu) against the FP64 oracle.

Inputs and weights are rounded to bfloat16 first; the FP64 oracle (oracle/conv.py) then sees the
very values the tensor cores multiply, so the only difference left is the FP32 accumulation:
max |kernel - oracle| <= 1e-4 * max |oracle| for the forward pass (FP32 copy before the ReLU),
the data gradient (with the ReLU mask of the layer input) and the weight and bias gradients.
Shapes cover every layer of the network (channels 2..128, strides 1 and 2) plus odd sizes.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import conv as OC

pytestmark = pytest.mark.gpu
TOL = 1e-4

# (batch, input size x y z, c_in, c_out, stride)
CASES = [(2, (10, 9, 8), 2, 16, 2), (1, (12, 10, 8), 16, 32, 2), (2, (7, 6, 5), 32, 64, 1),
         (1, (9, 7, 6), 64, 128, 2), (1, (6, 6, 4), 128, 64, 1), (2, (6, 6, 4), 64, 3, 1), (1, (5, 4, 3), 3, 8, 1)]


def _setup(case, seed):
    torch = pytest.importorskip("torch")
    from skmimageregistration_b200 import warmstart as W
    B, size, ci, co, s = case
    rng = np.random.default_rng(seed)
    x = OC.bf16_round(np.abs(rng.normal(size=(B, size[2], size[1], size[0], ci))) * (rng.uniform(size=(B, size[2], size[1], size[0], ci)) > 0.3))
    w = rng.normal(0, 0.2, (co, 27, ci))
    b = rng.normal(0, 0.1, co)
    layer = W.ConvLayer(torch, ci, co, s, True, rng)
    layer.load(w.reshape(co, -1), b)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    layer.pack(stream)
    wq = OC.bf16_round(w)
    xt = torch.tensor(x.astype(np.float32), device="cuda").to(torch.bfloat16).contiguous()
    return torch, W, layer, x, wq, b, xt, stream


def _close(got, ref):
    return float(np.max(np.abs(got - ref)) / max(np.max(np.abs(ref)), 1e-30))


@pytest.mark.parametrize("case", CASES)
def test_forward_matches_oracle(case):
    torch, W, L, x, wq, b, xt, stream = _setup(case, 1)
    B, size, ci, co, s = case
    osz = W.out_size(size, s)
    y = torch.empty((B, osz[2], osz[1], osz[0], co), dtype=torch.bfloat16, device="cuda")
    y32 = torch.empty(y.shape, dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    d = L.desc(B, size)
    assert W._lib().skm_conv3d_forward(C.byref(d), W._p(xt), W._p(L.wf), W._p(L.b), 1, W._p(y), W._p(y32), W._p(err),
                                       stream) == 0
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref = OC.forward(x, wq, b, s)
    assert _close(y32.cpu().numpy(), ref) <= TOL
    relu = np.maximum(y32.cpu().numpy(), 0.0)
    assert np.allclose(y.float().cpu().numpy(), relu, rtol=1e-2, atol=1e-6)        # bf16 of the ReLU output


@pytest.mark.parametrize("case", CASES)
def test_backward_data_matches_oracle(case):
    torch, W, L, x, wq, b, xt, stream = _setup(case, 2)
    B, size, ci, co, s = case
    osz = W.out_size(size, s)
    rng = np.random.default_rng(3)
    dy = OC.bf16_round(rng.normal(size=(B, osz[2], osz[1], osz[0], co)))
    dyt = torch.tensor(dy.astype(np.float32), device="cuda").to(torch.bfloat16).contiguous()
    dx = torch.empty_like(xt)
    dx32 = torch.empty(xt.shape, dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    d = L.desc(B, size)
    assert W._lib().skm_conv3d_backward_data(C.byref(d), W._p(dyt), W._p(L.wt), W._p(xt), W._p(dx), W._p(dx32),
                                             W._p(err), stream) == 0
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref = OC.backward_data(dy, wq, x.shape, s) * (x > 0)
    assert _close(dx32.cpu().numpy(), ref) <= TOL


@pytest.mark.parametrize("case", CASES)
def test_backward_weights_matches_oracle(case):
    torch, W, L, x, wq, b, xt, stream = _setup(case, 4)
    B, size, ci, co, s = case
    osz = W.out_size(size, s)
    rng = np.random.default_rng(5)
    dy = OC.bf16_round(rng.normal(size=(B, osz[2], osz[1], osz[0], co)))
    dyt = torch.tensor(dy.astype(np.float32), device="cuda").to(torch.bfloat16).contiguous()
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    d = L.desc(B, size)
    ws = W._lib().skm_conv3d_backward_weights_workspace(C.byref(d))
    work = torch.empty(ws, dtype=torch.uint8, device="cuda")
    assert W._lib().skm_conv3d_backward_weights(C.byref(d), W._p(xt), W._p(dyt), W._p(L.gw), W._p(L.gb), W._p(work),
                                                ws, W._p(err), stream) == 0
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    dw, db = OC.backward_weights(x, dy, s)
    assert _close(L.gw.cpu().numpy().reshape(co, 27, ci), dw) <= TOL
    assert _close(L.gb.cpu().numpy(), db) <= TOL


def test_training_on_the_gpu_reduces_the_loss():
    """Forward, backward and Adam of the whole network through the library's kernels: a few steps
    on a small batch fit it (the loss falls by more than half)."""
    torch = pytest.importorskip("torch")
    from skmimageregistration_b200 import warmstart as W
    rng = np.random.default_rng(0)
    net = W.WarmStartNet(seed=1)
    x = torch.tensor(rng.uniform(size=(4, 16, 32, 32, 2)).astype(np.float32), device="cuda").to(torch.bfloat16)
    target = torch.tensor(rng.normal(size=(4, 1 * 2 * 2 * 3)).astype(np.float32), device="cuda")
    losses = [net.train_step(x.contiguous(), target, lr=3e-3) for _ in range(60)]
    assert np.all(np.isfinite(losses))
    assert losses[-1] < 0.5 * losses[0], losses[::10]
