"""The FP64 convolution oracle (oracle/conv.py) against finite differences, on the CPU.

This pins the restatement the tcgen05 convolution kernels are checked against: its data and
weight gradients must equal central differences of the forward pass (FP64, 1e-6 relative).
"""
import numpy as np
import pytest

from oracle import conv as OC


@pytest.mark.parametrize("stride", [1, 2])
def test_oracle_gradients_match_finite_differences(stride):
    rng = np.random.default_rng(stride)
    x = rng.normal(size=(2, 5, 6, 7, 3))
    w = rng.normal(size=(4, 27, 3))
    b = rng.normal(size=4)
    y = OC.forward(x, w, b, stride)
    dy = rng.normal(size=y.shape)
    dx = OC.backward_data(dy, w, x.shape, stride)
    dw, db = OC.backward_weights(x, dy, stride)
    loss = lambda xx, ww, bb: float(np.sum(OC.forward(xx, ww, bb, stride) * dy))
    eps = 1e-6
    for _ in range(12):
        i = tuple(int(rng.integers(0, n)) for n in x.shape)
        xp, xm = x.copy(), x.copy()
        xp[i] += eps
        xm[i] -= eps
        fd = (loss(xp, w, b) - loss(xm, w, b)) / (2 * eps)
        assert abs(fd - dx[i]) <= 1e-6 * max(1.0, abs(fd))
        j = tuple(int(rng.integers(0, n)) for n in w.shape)
        wp, wm = w.copy(), w.copy()
        wp[j] += eps
        wm[j] -= eps
        fd = (loss(x, wp, b) - loss(x, wm, b)) / (2 * eps)
        assert abs(fd - dw[j]) <= 1e-6 * max(1.0, abs(fd))
    k = int(rng.integers(0, 4))
    bp, bm = b.copy(), b.copy()
    bp[k] += eps
    bm[k] -= eps
    assert abs((loss(x, w, bp) - loss(x, w, bm)) / (2 * eps) - db[k]) <= 1e-6 * max(1.0, abs(db[k]))


def test_output_size_and_bf16_rounding():
    assert OC.out_size(96, 2) == 48 and OC.out_size(7, 2) == 4 and OC.out_size(6, 1) == 6
    v = np.array([1.0, 1.00390625, 1.01171875, 1.001953125, -3.14159, 0.0])
    r = OC.bf16_round(v)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.015625      # halfway cases go to the even mantissa
    assert r[3] == 1.0 and abs(r[4] + 3.140625) < 1e-12 and r[5] == 0.0
