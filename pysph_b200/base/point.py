"""Point: a 3-vector of the API (S/base/point.pyx)."""
from __future__ import annotations

import math


class Point:
    __slots__ = ("x", "y", "z")

    def __init__(self, x=0.0, y=0.0, z=0.0):
        self.x, self.y, self.z = float(x), float(y), float(z)

    def set(self, x=0.0, y=0.0, z=0.0):
        self.x, self.y, self.z = float(x), float(y), float(z)

    def __sub__(self, o):
        return Point(self.x - o.x, self.y - o.y, self.z - o.z)

    def __add__(self, o):
        return Point(self.x + o.x, self.y + o.y, self.z + o.z)

    def dot(self, o):
        return self.x * o.x + self.y * o.y + self.z * o.z

    def norm(self):
        """Squared length, as the reference's Point.norm."""
        return self.x * self.x + self.y * self.y + self.z * self.z

    def length(self):
        return math.sqrt(self.norm())

    def asarray(self):
        return [self.x, self.y, self.z]

    def __repr__(self):
        return f"Point({self.x}, {self.y}, {self.z})"
