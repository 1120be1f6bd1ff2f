"""FP64 CPU restatement of the warm-start network's 3-D convolutions (test infrastructure only).

The reference has no learned component, so there is nothing of it to follow here: this is the
textbook definition of a 3x3x3 convolution with zero padding 1 and stride s (cross-correlation, as
deep-learning frameworks define it), its data gradient and its weight gradient, written with numpy
so that the CUDA kernels of skm_conv.cu can be checked against it.  Layouts match the kernels:
activations channels-last (B, Z, Y, X, C), weights (C_out, 27, C_in) with tap = 9 kz + 3 ky + kx.
Imported only by tests/.
"""
from __future__ import annotations

import numpy as np


def out_size(n, stride):
    return (n - 1) // stride + 1


def _taps():
    for kz in range(3):
        for ky in range(3):
            for kx in range(3):
                yield 9 * kz + 3 * ky + kx, kz, ky, kx


def forward(x, w, b=None, stride=1):
    """y[b, z, y, x, o] = sum_{tap, c} x[b, z s + kz - 1, y s + ky - 1, x s + kx - 1, c] w[o, tap, c] + b[o]."""
    x = np.asarray(x, np.float64)
    w = np.asarray(w, np.float64)
    B, Z, Y, X, Ci = x.shape
    Co = w.shape[0]
    Zo, Yo, Xo = out_size(Z, stride), out_size(Y, stride), out_size(X, stride)
    xp = np.zeros((B, Z + 2, Y + 2, X + 2, Ci))
    xp[:, 1:-1, 1:-1, 1:-1] = x
    y = np.zeros((B, Zo, Yo, Xo, Co))
    for t, kz, ky, kx in _taps():
        sl = xp[:, kz:kz + stride * (Zo - 1) + 1:stride, ky:ky + stride * (Yo - 1) + 1:stride,
                kx:kx + stride * (Xo - 1) + 1:stride]
        y += np.einsum("bzyxc,oc->bzyxo", sl, w[:, t, :])
    if b is not None:
        y += np.asarray(b, np.float64)
    return y


def backward_data(dy, w, in_shape, stride=1):
    """dx = d(sum y * dy)/dx for y = forward(x, w) (the transposed convolution)."""
    dy = np.asarray(dy, np.float64)
    w = np.asarray(w, np.float64)
    B, Z, Y, X, Ci = in_shape
    _, Zo, Yo, Xo, Co = dy.shape
    dxp = np.zeros((B, Z + 2, Y + 2, X + 2, Ci))
    for t, kz, ky, kx in _taps():
        dxp[:, kz:kz + stride * (Zo - 1) + 1:stride, ky:ky + stride * (Yo - 1) + 1:stride,
            kx:kx + stride * (Xo - 1) + 1:stride] += np.einsum("bzyxo,oc->bzyxc", dy, w[:, t, :])
    return dxp[:, 1:-1, 1:-1, 1:-1]


def backward_weights(x, dy, stride=1):
    """dw[o, tap, c] = d(sum y * dy)/dw and db[o] = sum dy for y = forward(x, w, b)."""
    x = np.asarray(x, np.float64)
    dy = np.asarray(dy, np.float64)
    B, Z, Y, X, Ci = x.shape
    _, Zo, Yo, Xo, Co = dy.shape
    xp = np.zeros((B, Z + 2, Y + 2, X + 2, Ci))
    xp[:, 1:-1, 1:-1, 1:-1] = x
    dw = np.zeros((Co, 27, Ci))
    for t, kz, ky, kx in _taps():
        sl = xp[:, kz:kz + stride * (Zo - 1) + 1:stride, ky:ky + stride * (Yo - 1) + 1:stride,
                kx:kx + stride * (Xo - 1) + 1:stride]
        dw[:, t, :] = np.einsum("bzyxo,bzyxc->oc", dy, sl)
    return dw, dy.sum(axis=(0, 1, 2, 3))


def bf16_round(a):
    """Round to the nearest bfloat16 (ties to even), as float64: the values the kernels read."""
    f = np.asarray(a, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)
