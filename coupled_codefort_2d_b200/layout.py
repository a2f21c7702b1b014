"""Field layout shared by the host API and the C ABI.

Every field is stored exactly as the Fortran callers of FUGU-2D allocate it
(``src/main.f90:97-103``): column-major, ``nh = 2`` ghost layers, custom
lower bounds.  A numpy array of the shape below in Fortran order *is* the
host buffer the C ABI reads (its first element is the lower-bound element).

=========  ============================  ==============  =================
kind       Fortran bounds                numpy shape     element (i, j)
=========  ============================  ==============  =================
``cell``   (1-nh:nx+nh, 1-nh:ny+nh)      (nx+4, ny+4)    ``a[i+1, j+1]``
``u``      (0-nh:nx+nh, 1-nh:ny+nh)      (nx+5, ny+4)    ``a[i+2, j+1]``
``v``      (1-nh:nx+nh, 0-nh:ny+nh)      (nx+4, ny+5)    ``a[i+1, j+2]``
``vert``   (0-nh:nx+nh, 0-nh:ny+nh)      (nx+5, ny+5)    ``a[i+2, j+2]``
=========  ============================  ==============  =================
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

NH = 2
KINDS = ("cell", "u", "v", "vert")
# lower-bound offsets (i0, j0): element (i, j) lives at a[i - i0, j - j0]
_LB = {"cell": (-1, -1), "u": (-2, -1), "v": (-1, -2), "vert": (-2, -2)}


@dataclass(frozen=True)
class Grid:
    """Single-rank Cartesian grid (``mod_mpi.f90:60-107`` with one process)."""

    nx: int
    ny: int
    Lx: float = 1.0
    Ly: float = 1.0
    periodic_x: bool = False
    periodic_y: bool = False

    @property
    def dx(self) -> float:
        return self.Lx / float(self.nx)

    @property
    def dy(self) -> float:
        return self.Ly / float(self.ny)

    def shape(self, kind: str) -> tuple[int, int]:
        nx, ny = self.nx, self.ny
        return {
            "cell": (nx + 4, ny + 4),
            "u": (nx + 5, ny + 4),
            "v": (nx + 4, ny + 5),
            "vert": (nx + 5, ny + 5),
        }[kind]

    def zeros(self, kind: str) -> np.ndarray:
        return np.zeros(self.shape(kind), dtype=np.float64, order="F")

    def full(self, kind: str, value: float) -> np.ndarray:
        return np.full(self.shape(kind), value, dtype=np.float64, order="F")

    @property
    def ncells(self) -> int:
        return self.nx * self.ny


def at(a: np.ndarray, kind: str, i, j):
    """Element / slice (i, j) of a field in Fortran index space."""
    i0, j0 = _LB[kind]
    if isinstance(i, slice):
        i = slice(i.start - i0, i.stop - i0 + 1)  # inclusive Fortran range
    else:
        i = i - i0
    if isinstance(j, slice):
        j = slice(j.start - j0, j.stop - j0 + 1)
    else:
        j = j - j0
    return a[i, j]


def interior(a: np.ndarray, kind: str, g: Grid) -> np.ndarray:
    """Owned unknowns: cells 1..nx x 1..ny; u faces 1..iu_max x 1..ny;
    v faces 1..nx x 1..jv_max (``mod_bicgstab2.f90:44-48``)."""
    nx, ny = g.nx, g.ny
    if kind == "cell":
        return at(a, kind, slice(1, nx), slice(1, ny))
    if kind == "u":
        imax = nx if g.periodic_x else nx - 1
        return at(a, kind, slice(1, imax), slice(1, ny))
    if kind == "v":
        jmax = ny if g.periodic_y else ny - 1
        return at(a, kind, slice(1, nx), slice(1, jmax))
    raise ValueError(kind)


def as_fortran(a: np.ndarray, g: Grid, kind: str) -> np.ndarray:
    """Validate a host buffer: float64, Fortran-contiguous, right shape."""
    if a.dtype != np.float64 or not a.flags.f_contiguous or a.shape != g.shape(kind):
        raise ValueError(
            f"field of kind {kind!r} must be a Fortran-ordered float64 array of shape "
            f"{g.shape(kind)}, got {a.dtype} {a.shape} f_contiguous={a.flags.f_contiguous}"
        )
    return a
