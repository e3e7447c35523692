"""Axis-aligned geometry primitives for the FDTD setup API.

The reference passes pyvista objects (``pv.Cube``, ``pv.Rectangle``, ``pv.Line``)
into ``FDTD_Solver`` and reads only their ``points`` (plus ``n_cells`` and
``faces`` as sanity checks, rfnetwork/solver.py:1092-1093, 1117, 1908).
These classes carry the same attributes for the shapes the FDTD setup
supports: boxes (dielectrics, conductors, the solve box), rectangles
(conductor sheets, port faces, current-probe faces) and lines (voltage
probes). Coordinates are in inches, as in the reference.
"""
from __future__ import annotations

import numpy as np


class Box:
    """Axis-aligned box; stands in for ``pv.Cube(center, x_length, y_length, z_length)``."""

    def __init__(self, center=(0.0, 0.0, 0.0), x_length=1.0, y_length=1.0, z_length=1.0, bounds=None):
        if bounds is not None:
            lo = np.array(bounds[0::2], dtype=float)
            hi = np.array(bounds[1::2], dtype=float)
        else:
            c = np.asarray(center, dtype=float)
            half = np.array([x_length, y_length, z_length], dtype=float) / 2
            lo, hi = c - half, c + half
        self.lo, self.hi = lo, hi
        corners = [[x, y, z] for x in (lo[0], hi[0]) for y in (lo[1], hi[1]) for z in (lo[2], hi[2])]
        self.points = np.array(corners, dtype=np.float32)
        # a closed box surface has 6 faces (the reference rejects dielectrics with more)
        self.n_cells = 6
        self.faces = np.array([4] * 6)

    @property
    def bounds(self):
        return (self.lo[0], self.hi[0], self.lo[1], self.hi[1], self.lo[2], self.hi[2])

    def implicit_distance(self, pts: np.ndarray) -> np.ndarray:
        """Signed distance from points (..., 3) to the box surface, negative inside."""
        lo = np.min(self.points, axis=0).astype(float)
        hi = np.max(self.points, axis=0).astype(float)
        d = np.maximum(lo - pts, pts - hi)
        outside = np.linalg.norm(np.maximum(d, 0.0), axis=-1)
        inside = np.minimum(np.max(d, axis=-1), 0.0)
        return outside + inside


class Rectangle:
    """Axis-aligned rectangle from three corner points; stands in for ``pv.Rectangle``.

    The fourth corner is ``p0 + p2 - p1``, as for pyvista's three-point form.
    """

    def __init__(self, points):
        p = np.asarray(points, dtype=float)
        if p.shape != (3, 3):
            raise ValueError("Rectangle needs three corner points")
        p3 = p[0] + p[2] - p[1]
        self.points = np.array([p[0], p[1], p[2], p3], dtype=np.float32)
        self.n_cells = 1
        self.faces = np.array([4, 0, 1, 2, 3])

    @property
    def bounds(self):
        lo, hi = np.min(self.points, axis=0), np.max(self.points, axis=0)
        return (lo[0], hi[0], lo[1], hi[1], lo[2], hi[2])


class Line:
    """Straight line between two points; stands in for ``pv.Line(p1, p2)``."""

    def __init__(self, p1, p2):
        self.points = np.array([p1, p2], dtype=np.float32)
        self.n_cells = 1


def is_object_surface(obj) -> bool:
    """True for a 2D object (rfnetwork/utils_mesh.py:166-177)."""
    x0, x1, y0, y1, z0, z1 = obj.bounds
    axis_len = np.abs(np.diff([[x0, y0, z0], [x1, y1, z1]], axis=0))
    return int(np.count_nonzero(axis_len > 1e-12)) == 2


def points_in_rectangle(points: np.ndarray, rect: Rectangle, tol: float) -> np.ndarray:
    """Inclusion test for grid points on an axis-aligned rectangle.

    Points on the rectangle's plane and inside its bounds, edges included
    (the reference's angle-sum test keeps edge points through its ``d_min``
    correction, rfnetwork/utils_mesh.py:383-525).
    """
    lo = np.min(rect.points, axis=0).astype(float)
    hi = np.max(rect.points, axis=0).astype(float)
    p = np.asarray(points, dtype=float)
    return np.all((p >= lo - tol) & (p <= hi + tol), axis=-1)
