"""Registration problem description: images, control-point grid and kernel.

This is the ITK-free restatement of what the reference's ITK glue hands to the
evaluator (itkTransformAdapter.hxx:386-462): the moving image's B-spline
coefficients, the fixed image, the control-point grid of
``TransformAdapter::ComputeControlPointImage`` (itkTransformAdapter.hxx:246-308)
and the kernel parameters.  Arrays are numpy, x-fastest (shape (Z, Y, X) in 3-D,
(Y, X) in 2-D), matching the reference's linear index x + X*(y + Y*z).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field as dc_field
from typing import Optional

import numpy as np

from .abi import EvaluatorDesc, Geometry, dptr


def control_point_grid(size, spacing, origin, sigma):
    """ComputeControlPointImage (itkTransformAdapter.hxx:246-308).

    cp spacing = sigma per axis; cp size = ceil(|upper_extent - lower_extent| / sigma);
    the cp grid is then centred: origin + |upper_extent - cp_upper_extent| / 2.
    Returns (cp_size, cp_spacing, cp_origin) as lists.
    """
    D = len(size)
    sigma = [float(sigma)] * D if np.isscalar(sigma) else [float(s) for s in sigma]
    lower = [float(origin[d]) for d in range(D)]
    upper = [float(origin[d]) + (int(size[d]) - 1) * float(spacing[d]) for d in range(D)]
    cp_size = [int(math.ceil(abs((upper[d] - lower[d]) / sigma[d]))) for d in range(D)]
    cp_upper = [float(origin[d]) + (cp_size[d] - 1) * sigma[d] for d in range(D)]
    cp_origin = [float(origin[d]) + abs(upper[d] - cp_upper[d]) / 2.0 for d in range(D)]
    return cp_size, sigma, cp_origin


def flat_to_aos(params, D):
    """Planar parameters [d*C + i] (itkTransformAdapter.hxx:202-236) -> AoS (C, D)."""
    p = np.asarray(params, dtype=np.float64)
    return np.ascontiguousarray(p.reshape(D, -1).T)


def aos_to_flat(cp):
    """AoS (C, D) control points -> planar parameters."""
    return np.ascontiguousarray(np.asarray(cp, dtype=np.float64).T.reshape(-1))


@dataclass
class Problem:
    """All inputs of one GpuKernelEvaluator (GpuEvaluator.h:147-154)."""

    fixed: np.ndarray                      # (Z,Y,X) or (Y,X) float64
    moving_coefficients: np.ndarray        # (Z+3,Y+3,X+3) or (Y+3,X+3) float64
    spacing: tuple
    origin: tuple
    sigma_c0: float
    sigma_c4: float
    cp_spacing: float                      # physical units
    subsample: int = 1
    subsample_neighborhood: int = 1
    weight_image: Optional[np.ndarray] = None     # non-stationary kernel (Kernel.h:105-117)
    weight_tensor: Optional[np.ndarray] = None    # anisotropic kernel, (..., D, D)
    maximum_weight: float = 0.0
    maximum_eigenvalue_covariance: Optional[np.ndarray] = None
    moving_origin: Optional[tuple] = None
    moving_spacing: Optional[tuple] = None
    _keep: list = dc_field(default_factory=list, repr=False)

    def __post_init__(self):
        self.fixed = np.ascontiguousarray(self.fixed, dtype=np.float64)
        self.moving_coefficients = np.ascontiguousarray(self.moving_coefficients, dtype=np.float64)
        self.D = self.fixed.ndim
        assert self.D in (2, 3)
        self.size = tuple(reversed(self.fixed.shape))          # (X, Y[, Z])
        self.cp_size, self.cp_sp, self.cp_origin = control_point_grid(
            self.size, self.spacing, self.origin, self.cp_spacing)
        self.C = int(np.prod(self.cp_size))
        if self.weight_image is not None:
            self.weight_image = np.ascontiguousarray(self.weight_image, dtype=np.float64)
            if self.maximum_weight == 0.0:
                self.maximum_weight = float(self.weight_image.max())   # SetWeightingImage
        if self.weight_tensor is not None:
            self.weight_tensor = np.ascontiguousarray(self.weight_tensor, dtype=np.float64)
            if self.maximum_eigenvalue_covariance is None:
                flat = self.weight_tensor.reshape(-1, self.D, self.D)
                ev = np.linalg.eigvalsh(flat)[:, -1]
                k = int(np.argmax(np.abs(ev)))                        # SetWeightingTensor
                self.maximum_eigenvalue_covariance = flat[k].copy()
                self.maximum_weight = float(abs(ev[k]))

    @property
    def num_parameters(self):
        return self.C * self.D

    @property
    def n_texels(self):
        return int(np.prod(self.size))

    def fixed_geometry(self):
        return Geometry.make(self.size, self.origin, self.spacing)

    def moving_geometry(self):
        return Geometry.make(self.size, self.moving_origin or self.origin,
                             self.moving_spacing or self.spacing)

    def cp_geometry(self):
        return Geometry.make(self.cp_size, self.cp_origin, self.cp_sp)

    def desc(self) -> EvaluatorDesc:
        """The C descriptor; host arrays stay owned by this object."""
        d = EvaluatorDesc()
        d.dimensions = self.D
        d.num_parameters = self.num_parameters
        d.subsample = int(self.subsample)
        d.subsample_neighborhood = int(self.subsample_neighborhood)
        d.sigma_c0 = float(self.sigma_c0)
        d.sigma_c4 = float(self.sigma_c4)
        d.use_weight_image = int(self.weight_image is not None)
        d.maximum_weight = float(self.maximum_weight)
        if self.weight_image is not None:
            d.weight_image = dptr(self.weight_image)
            d.weight_image_geometry = Geometry.make(tuple(reversed(self.weight_image.shape)),
                                                    self.origin, self.spacing)
        else:
            d.weight_image = None
            d.weight_image_geometry = Geometry.make([1] * self.D)
        d.use_weight_tensor = int(self.weight_tensor is not None)
        mc = np.zeros(9)
        if self.maximum_eigenvalue_covariance is not None:
            mc[: self.D * self.D] = np.asarray(self.maximum_eigenvalue_covariance).reshape(-1)
        for i in range(9):
            d.maximum_eigenvalue_covariance[i] = float(mc[i])
        if self.weight_tensor is not None:
            d.weight_tensor = dptr(self.weight_tensor)
            d.weight_tensor_geometry = Geometry.make(
                tuple(reversed(self.weight_tensor.shape[: self.D])), self.origin, self.spacing)
        else:
            d.weight_tensor = None
            d.weight_tensor_geometry = Geometry.make([1] * self.D)
        d.moving_coefficients = dptr(self.moving_coefficients)
        d.moving_geometry = self.moving_geometry()
        d.fixed_image = dptr(self.fixed)
        d.fixed_geometry = self.fixed_geometry()
        d.cp_geometry = self.cp_geometry()
        d.cpw_geometry = self.cp_geometry()
        self._keep = [self.fixed, self.moving_coefficients, self.weight_image, self.weight_tensor]
        return d
