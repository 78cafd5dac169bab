"""SPH kernel objects of the API (S/base/kernels.pyx:283-454).

CubicSplineKernel identifies the kernel the CUDA pair kernels evaluate (the
cubic spline of Monaghan 1992); its host-side function / gradient methods
evaluate single pairs for inspection and tests, with the reference's
formulas and normalisation (fac = 10/(7 pi h^2) in 2D, 1/(pi h^3) in 3D).
"""
from __future__ import annotations

import math

from .point import Point

CUBIC_SPLINE = 1   # kernel type id (S/base/kernels.pyx:33-44)


class KernelBase:
    def __init__(self, dim: int = 1, constant_h: float = -1):
        self.dim = dim
        self.constant_h = constant_h
        self.fac = self._fac(1.0)

    def radius(self) -> float:
        raise NotImplementedError

    def dimension(self) -> int:
        return self.dim

    def _fac(self, h):
        raise NotImplementedError


class CubicSplineKernel(KernelBase):
    """W(q) = fac {1 - 1.5 q^2 (1 - q/2), q <= 1; (2-q)^3 / 4, q <= 2; 0}."""

    def _fac(self, h):
        if self.dim == 1:
            return (2.0 / 3.0) / h
        if self.dim == 2:
            return 10 / (7 * math.pi) / (h * h)
        if self.dim == 3:
            return 1.0 / math.pi / (h * h * h)
        raise ValueError("dim must be 1, 2 or 3")

    def py_fac(self, h):
        return self._fac(h)

    def radius(self) -> float:
        return 2.0

    def get_type(self):
        return CUBIC_SPLINE

    def _h_dim(self, h):
        return 1 / h ** self.dim

    def py_function(self, pa: Point, pb: Point, h: float) -> float:
        rab = math.sqrt((pa.x - pb.x) ** 2 + (pa.y - pb.y) ** 2 + (pa.z - pb.z) ** 2)
        q = rab / h
        fac = self._h_dim(h) * self.fac
        if q > 2.0:
            val = 0.0
        elif q > 1.0:
            val = 0.25 * (2 - q) ** 3
        else:
            val = 1 - 1.5 * (q * q) * (1 - 0.5 * q)
        return val * fac

    def py_gradient(self, pa: Point, pb: Point, h: float, grad: Point):
        rab = math.sqrt((pa.x - pb.x) ** 2 + (pa.y - pb.y) ** 2 + (pa.z - pb.z) ** 2)
        q = rab / h
        fac = self._h_dim(h) * self.fac
        val = 0.0
        if q > 2.0:
            pass
        elif q >= 1.0:
            val = -0.75 * (2 - q) * (2 - q) / (h * rab)
        elif q > 1e-14:
            val = 3.0 * (0.75 * q - 1) / (h * h)
        grad.x = (pa.x - pb.x) * (val * fac)
        grad.y = (pa.y - pb.y) * (val * fac)
        grad.z = (pa.z - pb.z) * (val * fac)
