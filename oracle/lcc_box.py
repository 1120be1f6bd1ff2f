"""FP64 oracle of the box-window LCC -- test infrastructure only (tests/ import it as the checker).

The box-window local correlation is an extension beside the reference's LCC: the reference weights
the neighbours of a sample by (1 - (r/s)^10)^2 over the kernel support (include/cuda/
GpuEvaluatorLCC.cu:28-35,94-191); here every texel is a window centre and its window is the
(2r+1)^D box around it (r = 2: 5^3 in 3-D), clipped at the image border, over the texels whose
warped position is inside the moving image.  No reference code computes it, so parity is pinned
by finite differences of this restatement (tests/test_oracle_lcc_box.py) and the CUDA path is
checked against it.

Per counted centre x (inside, and both window variances above 1e-12 of their raw second moments,
so that flat windows are left out however their sums round):
    cov = S_fm - S_f S_m / n,  vf = S_ff - S_f^2 / n,  vm = S_mm - S_m^2 / n
    lcc_x = cov^2 / (vf vm)
    value = -(1 / count) sum_x lcc_x                      (the reference's LCC sign, cu:556-570)
d lcc_x / d m(y) = A_x (f(y) - mu_f(x)) + B_x (m(y) - mu_m(x)) for y in the window of x, with
A = 2 cov / (vf vm) and B = -2 cov^2 / (vf vm^2); the box is symmetric, so the coefficient of
texel y is a box sum over the centres around y:
    c(y) = -(f(y) S_A(y) + m(y) S_B(y) - S_E(y)),   E = A mu_f + B mu_m
and the derivative with respect to control point j is w_j / count * sum_y k(y, c_j) c(y) grad M(y),
the same control-point gather as the MSE and NCC derivatives.
"""
from __future__ import annotations

import numpy as np

from . import oracle as O

RADIUS = 2            # 5^D window
REL_EPS = 1e-12       # a window counts when vf > REL_EPS * S_ff and vm > REL_EPS * S_mm


def box_sum(a, r=RADIUS):
    """Sum over the (2r+1)^D box around every texel, clipped at the image border (separable)."""
    out = np.asarray(a, dtype=np.float64)
    for ax in range(out.ndim):
        n = out.shape[ax]
        pad = [(r, r) if k == ax else (0, 0) for k in range(out.ndim)]
        p = np.pad(out, pad)
        out = sum(np.take(p, np.arange(i, i + n), axis=ax) for i in range(2 * r + 1))
    return out


def window_terms(f, m, valid):
    """(measure, count, per-texel coefficient c) on image-shaped FP64 arrays."""
    v = valid.astype(np.float64)
    fv, mv = f * v, m * v
    n = box_sum(v)
    sf, sm = box_sum(fv), box_sum(mv)
    sff, smm, sfm = box_sum(fv * f), box_sum(mv * m), box_sum(fv * m)
    with np.errstate(divide="ignore", invalid="ignore"):
        muf = np.where(n > 0, sf / np.maximum(n, 1.0), 0.0)
        mum = np.where(n > 0, sm / np.maximum(n, 1.0), 0.0)
        vf = sff - sf * muf
        vm = smm - sm * mum
        cov = sfm - sf * mum
        counted = valid & (vf > REL_EPS * sff) & (vm > REL_EPS * smm)
        den = np.where(counted, vf * vm, 1.0)
        lcc = np.where(counted, cov * cov / den, 0.0)
        A = np.where(counted, 2.0 * cov / den, 0.0)
        B = np.where(counted, -2.0 * cov * cov / (den * np.where(counted, vm, 1.0)), 0.0)
    E = A * muf + B * mum
    sa, sb, se = box_sum(A), box_sum(B), box_sum(E)
    coef = np.where(valid, -(f * sa + m * sb - se), 0.0)
    count = int(counted.sum())
    measure = -float(lcc.sum()) / count if count else 0.0
    return measure, count, coef


def texel_positions(pb):
    """Global positions (N, D), components x, y[, z], texels in linear (x fastest) order."""
    shape = pb.fixed.shape                                  # (Z, Y, X) or (Y, X)
    idx = np.indices(shape).reshape(len(shape), -1)[::-1]   # x, y[, z]
    sp = np.asarray(pb.spacing, np.float64)[:, None]
    org = np.asarray(pb.origin, np.float64)[:, None]
    return np.ascontiguousarray((org + sp * idx).T)


def cp_positions(pb):
    g = pb.cp_geometry()
    D = pb.D
    size = [g.size[d] for d in range(D)]
    idx = np.indices(tuple(reversed(size))).reshape(D, -1)[::-1]
    org = np.array([g.origin[d] for d in range(D)])[:, None]
    sp = np.array([g.spacing[d] for d in range(D)])[:, None]
    return np.ascontiguousarray((org + sp * idx).T)


def evaluate(pb, cp, cpw, derivative=True):
    """(measure, count, derivative planar [d*C + j] or None) of the box-window LCC."""
    orc = O.Oracle(pb)
    u = orc.displacement_field(cp, cpw)
    orc.close()
    pos = texel_positions(pb)
    ins, m, gm = O.bspline_sample(pb.moving_coefficients, pb.moving_geometry(), pos + u)
    shape = pb.fixed.shape
    valid = (ins != 0).reshape(shape)
    mm = np.where(valid, m.reshape(shape), 0.0)
    measure, count, coef = window_terms(pb.fixed, mm, valid)
    if not derivative:
        return measure, count, None
    g = coef.reshape(-1)[:, None] * gm                      # (N, D); zero outside
    rows = np.nonzero(np.any(g != 0.0, axis=1))[0]
    cps = cp_positions(pb)
    C, D = pb.C, pb.D
    der = np.zeros(C * D)
    if count == 0 or rows.size == 0:
        return measure, count, der
    desc = pb.desc()
    chunk = max(1, 4_000_000 // rows.size)
    for j0 in range(0, C, chunk):
        j1 = min(C, j0 + chunk)
        p = np.repeat(pos[rows], j1 - j0, axis=0)
        q = np.tile(cps[j0:j1], (rows.size, 1))
        k = O.kernel_values(desc, q, p).reshape(rows.size, j1 - j0)
        acc = k.T @ g[rows]                                  # (cps, D)
        for d in range(D):
            der[d * C + j0:d * C + j1] = np.asarray(cpw[j0:j1]) * acc[:, d] / count
    return measure, count, der
