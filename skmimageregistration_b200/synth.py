"""Seeded synthetic registration pairs with the shapes of the benchmark workloads.

No public dataset is involved: every volume is generated from a seed.  Shapes and
value distributions follow the workload descriptions:

* ``blobs2d``    -- 256x256, 20 Gaussian blobs (sigma 8..30 px, amplitude U[0.2,1])
                    + N(0, 0.01), clipped to [0,1]; the moving image is the fixed one
                    warped by Wendland bumps on a 16 px grid with weights U[-4,4] px.
* ``ellipsoids3d`` -- 128x128x96, 6 random ellipsoids with intensities U[0,1] over a
                    smooth background + N(0, 0.02); sliding motion = 4-voxel shear of
                    opposite sign on either side of a random plane + smooth Wendland
                    displacement of up to 3 voxels.
* ``ct3d``       -- CT-like piecewise-constant ellipsoidal organs in [-1000, 1500]
                    + N(0, 20), 1.5 mm voxels, sliding displacement along a curved
                    boundary of up to 10 voxels.

Images are rescaled to [0, 1] as the reference driver does before registration
(src/SKMReg.cxx:87-90).  Arrays are (Z, Y, X) / (Y, X), float64.
"""
from __future__ import annotations

import numpy as np
from scipy import ndimage


def _rescale01(a):
    lo, hi = float(a.min()), float(a.max())
    return (a - lo) / (hi - lo) if hi > lo else np.zeros_like(a)


def _wendland(r):
    f = np.clip(1.0 - r, 0.0, None)
    return f ** 6 * (3.0 + 18.0 * r + 35.0 * r * r) / 3.0


def _warp(img, disp):
    """img sampled at x + disp(x) (disp: (D, ...) in voxels), cubic, mirrored borders."""
    grid = np.indices(img.shape, dtype=np.float64)
    coords = grid + disp
    return ndimage.map_coordinates(img, coords, order=3, mode="mirror")


def blobs2d(seed=0, shape=(256, 256)):
    rng = np.random.default_rng(seed)
    Y, X = shape
    yy, xx = np.mgrid[0:Y, 0:X].astype(np.float64)
    img = np.zeros(shape)
    for _ in range(20):
        cy, cx = rng.uniform(0, Y), rng.uniform(0, X)
        s = rng.uniform(8, 30)
        a = rng.uniform(0.2, 1.0)
        img += a * np.exp(-((yy - cy) ** 2 + (xx - cx) ** 2) / (2 * s * s))
    img += rng.normal(0, 0.01, shape)
    fixed = np.clip(img, 0.0, 1.0)
    # displacement: Wendland bumps on a 16 px grid, weights U[-4,4] px
    disp = np.zeros((2,) + shape)
    for gy in range(0, Y, 16):
        for gx in range(0, X, 16):
            w = rng.uniform(-4, 4, size=2)
            r = np.sqrt((yy - gy) ** 2 + (xx - gx) ** 2) / 16.0
            k = _wendland(r)
            disp[0] += w[1] * k
            disp[1] += w[0] * k
    moving = np.clip(_warp(fixed, disp), 0.0, 1.0)
    return _rescale01(fixed), _rescale01(moving), disp


def ellipsoids3d(seed=0, shape=(96, 128, 128)):
    """shape is (Z, Y, X); default 128x128x96 voxels (X, Y, Z)."""
    rng = np.random.default_rng(seed)
    Z, Y, X = shape
    zz, yy, xx = np.indices(shape, dtype=np.float64)
    bg = ndimage.gaussian_filter(rng.uniform(0, 0.3, shape), 12.0)
    img = bg.copy()
    for _ in range(6):
        c = [rng.uniform(0.2, 0.8) * n for n in shape]
        ax = [rng.uniform(0.08, 0.25) * n for n in shape]
        v = rng.uniform(0, 1)
        mask = ((zz - c[0]) / ax[0]) ** 2 + ((yy - c[1]) / ax[1]) ** 2 + ((xx - c[2]) / ax[2]) ** 2 <= 1.0
        img[mask] = v
    img = ndimage.gaussian_filter(img, 1.0) + rng.normal(0, 0.02, shape)
    fixed = img
    # sliding: 4-voxel shear of opposite sign across a random plane through the centre
    n = rng.normal(size=3)
    n /= np.linalg.norm(n)
    side = np.sign((zz - Z / 2) * n[0] + (yy - Y / 2) * n[1] + (xx - X / 2) * n[2])
    t = np.cross(n, [0.0, 0.0, 1.0] if abs(n[2]) < 0.9 else [1.0, 0.0, 0.0])
    t /= np.linalg.norm(t)
    disp = np.stack([side * 2.0 * t[i] for i in range(3)])        # +-2 -> 4-voxel relative shear
    # smooth Wendland displacement, up to 3 voxels
    for _ in range(8):
        c = [rng.uniform(0, nn) for nn in shape]
        r = np.sqrt((zz - c[0]) ** 2 + (yy - c[1]) ** 2 + (xx - c[2]) ** 2) / rng.uniform(16, 32)
        k = _wendland(r)
        disp += rng.uniform(-3, 3, size=3)[:, None, None, None] * k
    mag = np.sqrt((disp ** 2).sum(0)).max()
    moving = _warp(fixed, disp)
    return _rescale01(fixed), _rescale01(moving), disp


def ct3d(seed=0, shape=(160, 256, 256)):
    """CT-like volume, shape (Z, Y, X); default 256x256x160 voxels of 1.5 mm."""
    rng = np.random.default_rng(seed)
    Z, Y, X = shape
    zz, yy, xx = np.indices(shape, dtype=np.float32)
    img = np.full(shape, -1000.0, np.float32)
    body = ((zz - Z / 2) / (0.48 * Z)) ** 2 + ((yy - Y / 2) / (0.45 * Y)) ** 2 + ((xx - X / 2) / (0.47 * X)) ** 2 <= 1
    img[body] = 40.0
    for _ in range(10):
        c = [rng.uniform(0.25, 0.75) * n for n in shape]
        ax = [rng.uniform(0.06, 0.2) * n for n in shape]
        mask = ((zz - c[0]) / ax[0]) ** 2 + ((yy - c[1]) / ax[1]) ** 2 + ((xx - c[2]) / ax[2]) ** 2 <= 1.0
        img[mask & body] = rng.uniform(-900, 1500)
    img = img + rng.normal(0, 20, shape).astype(np.float32)
    fixed = img.astype(np.float64)
    # sliding along a curved boundary (a sphere), up to 10 voxels tangential motion
    r0 = 0.35 * min(shape)
    rr = np.sqrt((zz - Z / 2) ** 2 + (yy - Y / 2) ** 2 + (xx - X / 2) ** 2)
    inside = (rr < r0).astype(np.float64)
    amp = 10.0 * np.exp(-((rr - r0) / (0.3 * r0)) ** 2)
    disp = np.stack([amp * inside, np.zeros(shape), -amp * (1 - inside) * 0.5])
    moving = _warp(fixed, disp)
    return _rescale01(fixed), _rescale01(moving), disp
