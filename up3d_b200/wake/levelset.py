"""Implicit (level-set) representation of a straight ruled wake sheet, with
the reference's interface (pyfp3d/wake/levelset.py:1-225).

The sheet is swept from the trailing-edge polyline along a ruling
direction g.  A point x is written in the oblique frame of one TE segment
(a, v): x - a = u v + d g + s n, with n = unit(v x g) the "+" (upper)
normal.  u and d solve the 2 x 2 Gram system of (v, g); s = (x - a) . n.
The segment used for a point is the one nearest to it, counting the offset
s, the spanwise overshoot of u outside [0, 1] and a foot behind the TE
(d < 0).  Returned per point: s (signed offset), d (downstream distance
from the TE) and q (arclength along the TE polyline, not clamped).

Host numpy: evaluated once per mesh (and per incidence), not a hot path.
"""

from __future__ import annotations

from typing import Optional, Tuple

import numpy as np


class WakeLevelSet:
    """Signed offset / downstream / spanwise evaluation of a straight ruled
    wake surface (pyfp3d/wake/levelset.py:62-225): te_points (m >= 2, 3) or
    a single TE point (a long synthetic segment along span_hint), the
    physical wake direction, and optionally a different geometric ruling
    direction (sheet_direction)."""

    def __init__(self, te_points, direction, span_hint: Tuple[float, float, float] = (0.0, 0.0, 1.0),
                 extent: Optional[float] = None, sheet_direction=None):
        pts = np.atleast_2d(np.asarray(te_points, dtype=np.float64))
        if pts.shape[1] != 3:
            raise ValueError("te_points must be (m, 3)")
        if len(pts) == 1:
            axis = np.asarray(span_hint, dtype=np.float64)
            axis = axis / np.linalg.norm(axis)
            pts = np.vstack([pts[0] - 1e3 * axis, pts[0] + 1e3 * axis])
        self.te_points = pts
        self.extent = extent
        if sheet_direction is not None:
            sheet_direction = np.asarray(sheet_direction, dtype=np.float64)
            if sheet_direction.shape != (3,):
                raise ValueError("sheet_direction must be (3,)")
            if not np.any(sheet_direction):
                raise ValueError("sheet_direction must be nonzero")
        self._ruling = sheet_direction
        self._a = pts[:-1]
        self._v = pts[1:] - pts[:-1]
        vv = np.einsum("ij,ij->i", self._v, self._v)
        if np.any(vv <= 0.0):
            raise ValueError("degenerate TE segment (repeated points)")
        self._vv = vv
        self._vlen = np.sqrt(vv)
        self._q0 = np.concatenate([[0.0], np.cumsum(self._vlen)[:-1]])
        self.span_length = float(self._vlen.sum())
        self.update_direction(direction)

    @property
    def direction(self) -> np.ndarray:
        return self._dir.copy()

    @property
    def sheet_direction(self) -> Optional[np.ndarray]:
        return None if self._ruling is None else self._ruling.copy()

    def update_direction(self, new_direction) -> None:
        """Re-aims the sheet (an incidence change); the mesh is untouched."""
        d = np.asarray(new_direction, dtype=np.float64)
        norm = np.linalg.norm(d)
        if norm == 0.0:
            raise ValueError("direction must be nonzero")
        self._dir = d / norm
        g = self._dir if self._ruling is None else self._ruling / np.linalg.norm(self._ruling)
        self._g = g
        n = np.cross(self._v, g[None, :])
        nn = np.linalg.norm(n, axis=1)
        if np.any(nn < 1e-12 * self._vlen):
            raise ValueError("wake direction (near-)parallel to a TE segment")
        self._n = n / nn[:, None]
        self._vg = self._v @ g                   # v . g
        self._gram = self._vv - self._vg ** 2    # det of the (v, g) Gram matrix

    def _frame(self, points):
        """(u, d, s) per point and segment, and each point's segment."""
        x = np.atleast_2d(np.asarray(points, dtype=np.float64))
        rel = x[:, None, :] - self._a[None, :, :]
        rv = np.einsum("pns,ns->pn", rel, self._v)
        rg = rel @ self._g
        u = (rv - self._vg * rg) / self._gram
        d = (self._vv * rg - self._vg * rv) / self._gram
        s = np.einsum("pns,ns->pn", rel, self._n)
        over = np.maximum(0.0, np.maximum(-u, u - 1.0)) * self._vlen
        behind = np.minimum(0.0, d)
        seg = np.argmin(s ** 2 + over ** 2 + behind ** 2, axis=1)
        return u, d, s, seg

    def evaluate(self, points) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
        """(s, d, q) at points (n, 3)."""
        u, d, s, seg = self._frame(points)
        i = np.arange(len(seg))
        return s[i, seg], d[i, seg], self._q0[seg] + u[i, seg] * self._vlen[seg]

    def surface_normals(self, points) -> np.ndarray:
        """Unit "+" normal of the segment `evaluate` picks, per point."""
        return self._n[self._frame(points)[3]]
