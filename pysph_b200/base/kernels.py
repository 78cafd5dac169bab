"""SPH kernel objects of the API (S/base/kernels.pyx:283-640).

A kernel object tells the CUDA pair passes which smoothing kernel to
evaluate (get_type) and the neighbour radius (radius): the cubic spline
(2D and 3D), the quintic spline and the Wendland quintic (2D only, as in
the reference).  Their host-side function / gradient methods evaluate
single pairs for inspection and tests, with the reference's formulas and
normalisations, quirks included (see each class).
"""
from __future__ import annotations

import math

from .point import Point

# kernel type ids (S/base/kernels.pyx:31-40)
CUBIC_SPLINE = 1
QUINTIC_SPLINE = 3
WENDLAND_QUINTIC_SPLINE = 4


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


def _dist(pa: Point, pb: Point) -> float:
    return math.sqrt((pa.x - pb.x) ** 2 + (pa.y - pb.y) ** 2 + (pa.z - pb.z) ** 2)


class QuinticSplineKernel(KernelBase):
    """Quintic spline of Morris, Fox and Zhu (S/base/kernels.pyx:461-560),
    2D only, support 3h, fac = 7 / (478 pi h^2).  As in the reference, W
    adds (1 - q)^5 with weight 1 (not 15) and the gradient's value is
    +5 (3-q)^4 - 30 (2-q)^4 + 75 (1-q)^4, the opposite sign of dW/dq; the
    CUDA passes evaluate the same."""

    def _fac(self, h):
        if self.dim == 2:
            return 7.0 / (478 * math.pi * h * h)
        raise NotImplementedError("the quintic spline is 2D only")

    def py_fac(self, h):
        return self._fac(h)

    def radius(self) -> float:
        return 3.0

    def get_type(self):
        return QUINTIC_SPLINE

    def py_function(self, pa: Point, pb: Point, h: float) -> float:
        fac = self.fac / (h * h)
        q = _dist(pa, pb) / h
        if q > 3.0:
            return 0.0
        val = (3 - q) ** 5
        if q <= 2.0:
            val -= 6 * (2 - q) ** 5
            if q <= 1.0:
                val += (1 - q) ** 5
        return val * fac

    def py_gradient(self, pa: Point, pb: Point, h: float, grad: Point):
        fac = self.fac / (h * h)
        rab = _dist(pa, pb)
        q = rab / h
        val = 0.0
        if rab >= 1e-16:
            fac *= 1.0 / (h * rab)
            if q <= 3.0:
                val = 5 * (3 - q) ** 4
                if q <= 2.0:
                    val -= 30 * (2 - q) ** 4
                    if q <= 1.0:
                        val += 75 * (1 - q) ** 4
        grad.x = (pa.x - pb.x) * (val * fac)
        grad.y = (pa.y - pb.y) * (val * fac)
        grad.z = (pa.z - pb.z) * (val * fac)


class WendlandQuinticSplineKernel(KernelBase):
    """Wendland quintic (S/base/kernels.pyx:562-640), 2D only, support 2h,
    W = fac (1 - q/2)^4 (2q + 1).  The reference's _fac is written
    (7./4*PI*h*h), so fac = 7 pi h^2 / 4 (not 7 / (4 pi h^2)); kept, on
    the host and in the CUDA passes."""

    def _fac(self, h):
        if self.dim == 2:
            return 7.0 / 4 * math.pi * h * h
        raise NotImplementedError("the Wendland quintic is 2D only")

    def py_fac(self, h):
        return self._fac(h)

    def radius(self) -> float:
        return 2.0

    def get_type(self):
        return WENDLAND_QUINTIC_SPLINE

    def py_function(self, pa: Point, pb: Point, h: float) -> float:
        fac = self.fac / (h * h)
        q = _dist(pa, pb) / h
        if q > 2.0:
            return 0.0
        return (1 - 0.5 * q) ** 4 * (2 * q + 1) * fac

    def py_gradient(self, pa: Point, pb: Point, h: float, grad: Point):
        fac = self.fac / (h * h)
        rab = _dist(pa, pb)
        q = rab / h
        val = 0.0
        if rab >= 1e-16:
            fac *= 1.0 / (h * rab)
            if q <= 2.0:
                val = (1 - 0.5 * q) ** 3 * -5 * q
        grad.x = (pa.x - pb.x) * (val * fac)
        grad.y = (pa.y - pb.y) * (val * fac)
        grad.z = (pa.z - pb.z) * (val * fac)
