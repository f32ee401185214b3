"""Grids and boundary conditions of the dynamical core.

Mirrors the reference's mesh types: `RegularGrid` (src/Grids.jl:98-130),
`StretchedGrid` with its face generators (src/StretchedGrids.jl:117-400) and
the axis boundary kinds of `FieldBoundaryConditions`
(src/BoundaryConditions.jl:54-137): x and y periodic; z periodic or an
impermeable free-slip wall (`:wall`).

A field on a grid is stored as in the reference's `Field.data`: a
column-major (x fastest) array of (Nx+2Hx)(Ny+2Hy)(Nz+2Hz) Float64 values.
In numpy that is a C-ordered array of shape (Nz+2Hz, Ny+2Hy, Nx+2Hx),
indexed [k, j, i].
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Optional, Tuple

import numpy as np

PERIODIC = "periodic"
WALL = "wall"


@dataclass
class Grid:
    """A uniform or vertically stretched staggered (Arakawa-C) grid.

    `size` (Nx, Ny, Nz) interior cells, `extent` (Lx, Ly, Lz), `halo`
    (Hx, Hy, Hz) of the storage arrays, `origin`, `bc_z` ("periodic" or
    "wall"), and `zf` the Nz+1 interior face heights of a stretched column
    (None for uniform z).
    """

    size: Tuple[int, int, int]
    extent: Tuple[float, float, float]
    halo: Tuple[int, int, int] = (3, 3, 3)
    origin: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    bc_z: str = PERIODIC
    zf: Optional[np.ndarray] = field(default=None, repr=False)

    def __post_init__(self):
        nx, ny, nz = self.size
        if min(nx, ny, nz) <= 0:
            raise ValueError(f"size must be positive, got {self.size}")
        if self.bc_z not in (PERIODIC, WALL):
            raise ValueError(f"bc_z must be 'periodic' or 'wall', got {self.bc_z!r}")
        if self.zf is not None:
            self.zf = np.ascontiguousarray(self.zf, dtype=np.float64)
            if self.zf.shape != (nz + 1,):
                raise ValueError(f"zf must have Nz+1 = {nz + 1} entries, got {self.zf.shape}")
            if np.any(np.diff(self.zf) <= 0):
                raise ValueError("zf must be strictly increasing")

    # ---- shapes -------------------------------------------------------------
    @property
    def nx(self):
        return self.size[0]

    @property
    def ny(self):
        return self.size[1]

    @property
    def nz(self):
        return self.size[2]

    @property
    def stretched(self) -> bool:
        return self.zf is not None

    @property
    def storage_shape(self) -> Tuple[int, int, int]:
        """numpy shape (Nz+2Hz, Ny+2Hy, Nx+2Hx) of a storage array."""
        hx, hy, hz = self.halo
        return (self.nz + 2 * hz, self.ny + 2 * hy, self.nx + 2 * hx)

    @property
    def interior(self) -> Tuple[slice, slice, slice]:
        """numpy index of the interior of a storage array ([k, j, i])."""
        hx, hy, hz = self.halo
        return (slice(hz, hz + self.nz), slice(hy, hy + self.ny), slice(hx, hx + self.nx))

    @property
    def ncells(self) -> int:
        return self.nx * self.ny * self.nz

    @property
    def dx(self) -> float:
        return self.extent[0] / self.nx

    @property
    def dy(self) -> float:
        return self.extent[1] / self.ny

    @property
    def dz(self) -> float:
        return self.extent[2] / self.nz

    def zeros(self) -> np.ndarray:
        return np.zeros(self.storage_shape)

    # ---- node coordinates (src/Grids.jl:150-170) ------------------------------
    def xnodes(self, loc: str = "c") -> np.ndarray:
        i = np.arange(self.nx, dtype=np.float64)
        return self.origin[0] + ((i + 0.5) if loc != "fx" else i) * self.dx

    def ynodes(self, loc: str = "c") -> np.ndarray:
        j = np.arange(self.ny, dtype=np.float64)
        return self.origin[1] + ((j + 0.5) if loc != "fy" else j) * self.dy

    def znodes(self, loc: str = "c") -> np.ndarray:
        """Interior level heights: cell centres, or the bottom faces for loc='fz'."""
        if self.zf is None:
            k = np.arange(self.nz, dtype=np.float64)
            return self.origin[2] + ((k + 0.5) if loc != "fz" else k) * self.dz
        if loc == "fz":
            return self.zf[:-1].copy()
        return 0.5 * (self.zf[:-1] + self.zf[1:])

    def cell_thickness(self) -> np.ndarray:
        """Interior Δz_c (length Nz)."""
        if self.zf is None:
            return np.full(self.nz, self.dz)
        return np.diff(self.zf)


def regular_grid(size, extent, halo=(3, 3, 3), origin=(0.0, 0.0, 0.0), bc_z=PERIODIC) -> Grid:
    """`RegularGrid` (src/Grids.jl:98-117)."""
    return Grid(tuple(size), tuple(float(e) for e in extent), tuple(halo), tuple(origin), bc_z, None)


def tanh_faces(nz: int, lz: float, beta: float, z0: float = 0.0) -> np.ndarray:
    """Bottom-clustered tanh faces (`_faces_tanh`, src/StretchedGrids.jl:191-205):
    z_k = z0 + Lz (1 - tanh(β(1 - ξ_k)) / tanh β), ξ_k = (k-1)/Nz."""
    if beta <= 0:
        raise ValueError(f"tanh stretching β must be > 0, got {beta}")
    tb = math.tanh(beta)
    zf = np.empty(nz + 1)
    for k in range(nz + 1):
        xi = k / nz
        zf[k] = z0 + lz * (1 - math.tanh(beta * (1 - xi)) / tb)
    zf[0] = z0
    zf[nz] = z0 + lz
    return zf


def tanh_beta_for_first_cell(nz: int, lz: float, dz1: float) -> float:
    """The β of `tanh_faces` whose first cell is `dz1` thick (bisection)."""
    if not (0 < dz1 < lz / nz):
        raise ValueError("dz1 must lie in (0, Lz/Nz) for bottom clustering")
    lo, hi = 1e-8, 20.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        d = tanh_faces(nz, lz, mid)[1]
        if d > dz1:
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi)


def stretching_ratio(zf: np.ndarray) -> float:
    """Largest ratio of adjacent cell thicknesses (`grid_stretching_ratio`,
    src/StretchedGrids.jl:466-478)."""
    d = np.diff(zf)
    r = d[1:] / d[:-1]
    return float(np.max(np.maximum(r, 1 / r)))


def stretched_grid(size, extent, zf, halo=(3, 3, 3), origin=(0.0, 0.0, 0.0)) -> Grid:
    """`StretchedGrid(stretching = (:custom, zf))` with walls in z."""
    return Grid(tuple(size), tuple(float(e) for e in extent), tuple(halo), tuple(origin), WALL, np.asarray(zf))
