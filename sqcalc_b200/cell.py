"""Simulation cell: lattice vectors, reciprocal basis, LAMMPS bounds.

Host-side restatement of thatstar/sqcalc src/sqc_cell.f90.  Arrays use the
reference's Fortran layout flattened in memory order: ``a`` holds the three
lattice vectors one after the other (a(3,3) column major: a[i] is vector i),
``b`` the reciprocal vectors the same way, with a_i . b_j = 2 pi delta_ij.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

TWO_PI = 2.0 * math.acos(-1.0)


def _det3(m):
    # determinant3, src/sqc_cell.f90:131-137 (m[c][r] = m(r+1, c+1))
    M = lambda r, c: m[c - 1][r - 1]  # noqa: E731
    return (M(1, 1) * (M(2, 2) * M(3, 3) - M(2, 3) * M(3, 2))
            - M(1, 2) * (M(2, 1) * M(3, 3) - M(2, 3) * M(3, 1))
            + M(1, 3) * (M(2, 1) * M(3, 2) - M(2, 2) * M(3, 1)))


def inverse3(a):
    """inverse3 (src/sqc_cell.f90:139-152); a and the result in the column layout."""
    m = [[float(a[c][r]) for r in range(3)] for c in range(3)]
    M = lambda r, c: m[c - 1][r - 1]  # noqa: E731
    det = _det3(m)
    inv = [[0.0] * 3 for _ in range(3)]

    def put(r, c, v):
        inv[c - 1][r - 1] = v

    put(1, 1, (M(2, 2) * M(3, 3) - M(2, 3) * M(3, 2)))
    put(2, 1, -(M(2, 1) * M(3, 3) - M(2, 3) * M(3, 1)))
    put(3, 1, (M(2, 1) * M(3, 2) - M(2, 2) * M(3, 1)))
    put(1, 2, -(M(1, 2) * M(3, 3) - M(1, 3) * M(3, 2)))
    put(2, 2, (M(1, 1) * M(3, 3) - M(1, 3) * M(3, 1)))
    put(3, 2, -(M(1, 1) * M(3, 2) - M(1, 2) * M(3, 1)))
    put(1, 3, (M(1, 2) * M(2, 3) - M(1, 3) * M(2, 2)))
    put(2, 3, -(M(1, 1) * M(2, 3) - M(1, 3) * M(2, 1)))
    put(3, 3, (M(1, 1) * M(2, 2) - M(1, 2) * M(2, 1)))
    return np.array([[v / det for v in col] for col in inv])


@dataclass
class Cell:
    a: np.ndarray = field(default_factory=lambda: np.zeros((3, 3)))
    origin: np.ndarray = field(default_factory=lambda: np.zeros(3))

    @property
    def inv(self):
        return inverse3(self.a)

    @property
    def b(self):
        """b_j = 2 pi * row j of A^-1 (cell_setup, src/sqc_cell.f90:78-88)."""
        inv = self.inv  # inv[c][r] = A^-1(r+1, c+1)
        return np.array([[TWO_PI * inv[c][j] for c in range(3)] for j in range(3)])

    @property
    def volume(self):
        return abs(_det3(self.a))

    @classmethod
    def from_bounds(cls, lo, hi, tilt):
        """cell_init_from_bounds (src/sqc_cell.f90:38-63): LAMMPS bounding box to
        the restricted triclinic cell."""
        xy, xz, yz = (float(t) for t in tilt)
        xlo = lo[0] - min(0.0, xy, xz, xy + xz)
        xhi = hi[0] - max(0.0, xy, xz, xy + xz)
        ylo = lo[1] - min(0.0, yz)
        yhi = hi[1] - max(0.0, yz)
        zlo, zhi = lo[2], hi[2]
        a = np.array([[xhi - xlo, 0.0, 0.0], [xy, yhi - ylo, 0.0], [xz, yz, zhi - zlo]])
        return cls(a=a, origin=np.array([xlo, ylo, zlo], dtype=np.float64))

    @classmethod
    def cubic(cls, length):
        return cls(a=np.eye(3) * float(length), origin=np.zeros(3))

    def flat(self):
        """The nine numbers in the Fortran memory order of a(3,3)."""
        return np.ascontiguousarray(self.a, dtype=np.float64).reshape(9)
