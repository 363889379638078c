"""Curve discretisation, mirroring ImmersedBodies.jl's `src/curves.jl` (host only).

Only the curves the hot-path configurations use are mirrored: `Circle`,
`LineSegment` and affine transforms of them, with `partition` by count or
by target spacing and `panels_for(grid, curve)` = `Panels(grid, curve)`
(curves.jl:53-55, partition at spacing 2h).
"""
from __future__ import annotations

import math

import numpy as np

from .problem import MultiDomainGrid, Panels


class Curve:
    closed = False

    def arclength(self) -> float:
        raise NotImplementedError

    def partition_n(self, n: int) -> Panels:
        raise NotImplementedError


def partition(curve: Curve, n_or_ds) -> Panels:
    """partition(curve, n::Integer) / partition(curve, ds::AbstractFloat) (curves.jl:75-82)."""
    if isinstance(n_or_ds, (int, np.integer)):
        return curve.partition_n(int(n_or_ds))
    n = int(round(curve.arclength() / float(n_or_ds))) + (0 if curve.closed else 1)
    return curve.partition_n(n)


class LineSegment(Curve):
    """LineSegment((x1, y1), (x2, y2)) (curves.jl:176-196)."""

    closed = False

    def __init__(self, p1, p2):
        self.p1 = np.asarray(p1, dtype=float)
        self.p2 = np.asarray(p2, dtype=float)

    def arclength(self):
        return float(np.hypot(*(self.p2 - self.p1)))

    def partition_n(self, n):
        xb = np.column_stack([np.linspace(self.p1[0], self.p2[0], n), np.linspace(self.p1[1], self.p2[1], n)])
        return Panels(xb, np.full(n, self.arclength() / (n - 1)))


class Circle(Curve):
    """Circle(; r, center) (curves.jl:203-231)."""

    closed = True

    def __init__(self, r=1.0, center=(0.0, 0.0)):
        self.r = float(r)
        self.center = np.asarray(center, dtype=float)

    def arclength(self):
        return 2 * math.pi * self.r

    def partition_n(self, n):
        t = 2 * math.pi / n * np.arange(n)
        xs = self.center[0] + self.r * np.cos(t)
        ys = self.center[1] + self.r * np.sin(t)
        ds = math.hypot(xs[1] - xs[0], ys[1] - ys[0])
        return Panels(np.column_stack([xs, ys]), np.full(n, ds))


class Transformation:
    """Translation, rotation and uniform scale (curves.jl:91-134)."""

    def __init__(self, offset=(0.0, 0.0), rotation=None, scale=1.0):
        self.offset = np.asarray(offset, dtype=float)
        self.rotation = np.eye(2) if rotation is None else np.asarray(rotation, dtype=float)
        self.scale = float(scale)

    def apply(self, v):
        return self.offset + self.rotation @ (self.scale * np.asarray(v, dtype=float))

    def __call__(self, x):
        if isinstance(x, Curve):
            return TransformedCurve(x, self)
        return self.apply(x)


def translate(v) -> Transformation:
    return Transformation(offset=v)


def rotate(theta) -> Transformation:
    c, s = math.cos(theta), math.sin(theta)
    return Transformation(rotation=[[c, -s], [s, c]])


def scale(k) -> Transformation:
    return Transformation(scale=k)


class TransformedCurve(Curve):
    def __init__(self, base: Curve, transform: Transformation):
        self.base = base
        self.transform = transform
        self.closed = base.closed

    def arclength(self):
        return abs(self.transform.scale) * self.base.arclength()

    def partition_n(self, n):
        p = self.base.partition_n(n)
        xb = np.array([self.transform.apply(x) for x in p.xb])
        return Panels(xb, p.ds * self.transform.scale)


def panels_for(grid: MultiDomainGrid, curve: Curve) -> Panels:
    """Panels(grid, curve) = partition(curve, 2h) (curves.jl:53-55)."""
    return partition(curve, 2.0 * grid.base.h)
