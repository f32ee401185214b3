"""Open lateral faces: Dirichlet halos from boundary data and the single
global boundary mass-flux correction (src/boundary_conditions/open_boundary.jl).

    data = ProfileBoundaryData(u=5.0, v=0.0, w=0.0, theta=lambda z: 300.0 + 0.003 * z)
    obc = open_boundary_conditions(grid, data, x="open", y="periodic")
    sim.set_open_boundaries(obc)          # the step fills its halos from obc's planes
    obc.ledger                            # {"Q", "residual", "delta"} of the correction

A face is "open" when the normal velocity on it is prescribed from outside
the domain and the projection must leave it unchanged (`OpenBoundary`,
:485-531): on every halo fill the normal velocity's boundary face and the
layers beyond it, the tangential velocities and the scalars with data are
copied from plane buffers, every other field gets the zero-gradient mirror
(the Neumann condition that keeps the prescribed normal velocity through the
projection, Kim & Moin 1985).  The buffers hold the boundary data at the
storage points of the faces' halo slabs (`OpenPlane`, :72-161); the normal
velocity's boundary-face values are then made mass consistent by
`correct_boundary_mass_flux!` (:1024-1083): with every face's normal velocity
prescribed, the Neumann problem of the projection is solvable only when the
net boundary flux vanishes.

Built here: open x and/or y faces over a wall bottom and a wall (rigid-lid)
top, on the uniform Boussinesq core with the PCG projection; steady data
(`ProfileBoundaryData`, :336-408, and `FunctionBoundaryData` evaluated at one
time, :330-380); outflow `:dirichlet` (every point takes the data); normal
halo `:value`; scalar halo `:value` or `:mirror`; corrections `:uniform`,
`:outflow_only` and `:none`.  The buffers are static, so the correction is
applied once here (the reference applies the same correction to the same
data before every projection).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Callable, Dict, Optional

import numpy as np

from .grids import Grid, WALL

FIELDS = ("u", "v", "w", "theta")
_AXIS = {"west": (0, False), "east": (0, True), "south": (1, False), "north": (1, True)}
_NORMAL = {"u": 0, "v": 1, "w": 2, "theta": -1}
CORRECTIONS = ("uniform", "outflow_only", "none")


class ProfileBoundaryData:
    """Horizontally uniform, steady boundary data (`ProfileBoundaryData`,
    src/boundary_conditions/open_boundary.jl:336-355): each keyword is a
    number, a function of height `z -> value`, or a vector indexed by the
    storage z index (length Nz + 2Hz).  `w` defaults to zero; any other field
    with an open plane but no data raises ValueError."""

    def __init__(self, **fields):
        self.fields = dict(fields)

    def value(self, name, x, y, z, kstore):
        f = _data_for(self.fields, name, "ProfileBoundaryData")
        if callable(f):
            prof = np.array([float(f(zz)) for zz in z])
        elif np.ndim(f) == 0:
            prof = np.full(len(z), float(f))
        else:
            f = np.asarray(f, dtype=np.float64)
            if f.size <= kstore[-1]:
                raise ValueError(f"profile for {name} has {f.size} entries; a storage-indexed profile needs "
                                 f"at least {kstore[-1] + 1}")
            prof = f[kstore]
        return np.broadcast_to(prof[:, None, None], (len(z), len(y), len(x)))


class FunctionBoundaryData:
    """Analytic boundary data f(x, y, z, t) per field (`FunctionBoundaryData`,
    :330-380), evaluated at the storage points of the planes at the time `t`
    given to open_boundary_conditions (steady in the step)."""

    def __init__(self, t: float = 0.0, **fields):
        self.t = float(t)
        self.fields = dict(fields)

    def value(self, name, x, y, z, kstore):
        f = _data_for(self.fields, name, "FunctionBoundaryData")
        if not callable(f):
            return np.full((len(z), len(y), len(x)), float(f))
        Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
        return np.vectorize(lambda a, b, c: float(f(a, b, c, self.t)))(X, Y, Z)


def _data_for(fields, name, kind):
    """_data_for (:356-361): a field's data, zero for a missing w."""
    if name in fields:
        return fields[name]
    if name == "theta" and "θ" in fields:
        return fields["θ"]
    if name == "w":
        return 0.0
    raise ValueError(f"{kind} has no data for the open-boundary field {name} (it provides {sorted(fields)})")


@dataclass
class OpenPlane:
    """The boundary data of one field on one open face (`OpenPlane`, :72-161):
    `data` is the storage slab the face writes ([k, j, i] over the full
    storage extent of the two other axes and, along the face normal, the H
    halo layers plus, for the normal velocity of a west/south face, the
    boundary face itself, interior index 0), `start` its first storage index
    along the normal, `fluid` the faces that carry flow (interior tangential
    indices), `mode` "value" or "mirror"."""

    name: str
    side: str
    axis: int
    high: bool
    normal: bool
    mode: str
    start: int
    data: np.ndarray
    fluid: np.ndarray = field(repr=False)

    def face_layer(self, H):
        """Local index (along the normal) of the boundary face (_face_local, :163)."""
        return 0 if self.high else H


def _coord(x0, d, H, i0, staggered):
    """Coordinate of 0-based storage index i0 (_coord, :162-164, 1-based there)."""
    return x0 + (i0 - H + (0.0 if staggered else 0.5)) * d


class OpenBoundarySet:
    """Every plane of the open faces of one domain, the correction mode and
    the ledger of the last correction (`OpenBoundaryState`, :445-485)."""

    def __init__(self, grid: Grid, planes, correction: str, open_x: bool, open_y: bool):
        self.grid = grid
        self.planes = planes
        self.correction = correction
        self.open_x = open_x
        self.open_y = open_y
        self.ledger = {"Q": 0.0, "residual": 0.0, "delta": 0.0}

    def plane(self, name, side):
        for p in self.planes:
            if p.name == name and p.side == side:
                return p
        return None

    # ---- the mass-flux correction (correct_boundary_mass_flux!, :1024-1083) ----------
    def _face_terms(self, p):
        """(outward flux, outflow area, area) over the fluid faces of normal
        plane p (_face_sums, :994-1012), and the face values / areas."""
        g = self.grid
        hx, hy, hz = g.halo
        nx, ny, nz = g.size
        fl = p.face_layer(g.halo[p.axis])
        if p.axis == 0:
            vals = p.data[hz:hz + nz, hy:hy + ny, fl]                 # [k, j]
            area = g.dy * g.dz
        else:
            vals = p.data[hz:hz + nz, fl, hx:hx + nx]                 # [k, i]
            area = g.dx * g.dz
        s = 1.0 if p.high else -1.0
        f = p.fluid.T                                                  # [k, tangential]
        out = s * vals
        q = float(np.sum(np.where(f, out * area, 0.0)))
        ao = float(np.sum(np.where(f & (out > 0), area, 0.0)))
        aa = float(np.sum(np.where(f, area, 0.0)))
        return q, ao, aa

    def flux(self):
        """Net outward volume flux Q = sum u.n A over the open fluid faces
        (open_boundary_flux, :940-957)."""
        return sum(self._face_terms(p)[0] for p in self.planes if p.normal)

    def correct(self):
        """Remove the data's net outward flux from the normal velocities:
        delta = Q / (sum of A) subtracted from the outward normal velocity of
        every open fluid face (:uniform), or from the outflow faces only
        (:outflow_only, all faces when none flows out); :none records Q only.
        Returns delta."""
        g = self.grid
        Q = Aout = Aall = 0.0
        for p in self.planes:
            if p.normal:
                q, ao, aa = self._face_terms(p)
                Q += q
                Aout += ao
                Aall += aa
        delta = 0.0
        if self.correction != "none" and Q != 0.0:
            only_out = self.correction == "outflow_only"
            A = Aout if only_out else Aall
            if A == 0.0:
                only_out, A = False, Aall
            delta = Q / A
            hx, hy, hz = g.halo
            nx, ny, nz = g.size
            for p in self.planes:
                if not p.normal:
                    continue
                s = 1.0 if p.high else -1.0
                fl = p.face_layer(g.halo[p.axis])
                if p.axis == 0:
                    view = p.data[hz:hz + nz, hy:hy + ny, fl]
                else:
                    view = p.data[hz:hz + nz, fl, hx:hx + nx]
                sel = p.fluid.T.copy()
                if only_out:
                    sel &= (s * view) > 0
                view[sel] -= s * delta
        self.ledger = {"Q": Q, "residual": self.flux(), "delta": delta}
        return delta

    # ---- the device image ---------------------------------------------------------------
    def packed(self):
        """The planes as the arrays aeo_set_open takes: x planes
        [field][side][k][j][layer] (NZ x NY x (H+1)) and y planes
        [field][side][k][layer][i] (NZ x (H+1) x NX), field order u, v, w,
        theta, layer = storage index along the normal on the low side and
        storage index - (H + N) on the high side; and the per-field mode
        (0 value, 1 mirror)."""
        g = self.grid
        hx, hy, hz = g.halo
        NZ, NY, NX = g.storage_shape
        L = max(hx, hy) + 1
        xp = np.zeros((4, 2, NZ, NY, L))
        yp = np.zeros((4, 2, NZ, L, NX))
        modes = np.zeros(4, dtype=np.int32)
        for p in self.planes:
            f = FIELDS.index(p.name)
            side = 1 if p.high else 0
            if p.mode == "mirror":
                modes[f] = 1
                continue
            H = g.halo[p.axis]
            N = g.size[p.axis]
            off = p.start - (H + N) if p.high else p.start
            n = p.data.shape[2 - p.axis]
            if p.axis == 0:
                xp[f, side, :, :, off:off + n] = p.data
            else:
                yp[f, side, :, off:off + n, :] = p.data
        return np.ascontiguousarray(xp), np.ascontiguousarray(yp), modes


def open_boundary_conditions(grid: Grid, data, x: str = "open", y: str = "periodic",
                             fields=FIELDS, correction: str = "uniform", normal_halo: str = "value",
                             scalar_halo: str = "value", outflow: str = "dirichlet") -> OpenBoundarySet:
    """A box with open lateral faces fed by `data` (`open_boundary_conditions`,
    :532-638): `x` and `y` each "open" or "periodic" (both faces of an axis
    alike), bottom and top walls.  `fields` names the fields with boundary
    data (the three velocity components and theta); the planes are filled
    from `data` and the normal velocities corrected (`correction`).
    Raises ValueError for what is not built (an open top or bottom, the
    :odd normal halo, radiating outflow, the :inflow scalar halo)."""
    if x not in ("open", "periodic") or y not in ("open", "periodic"):
        raise ValueError("x and y are 'open' or 'periodic'")
    if x == "periodic" and y == "periodic":
        raise ValueError("no open face: give x = 'open' and/or y = 'open'")
    if grid.bc_z != WALL:
        raise ValueError("open lateral faces need wall bottom and top (bc_z = 'wall'); an open top is not built")
    if grid.stretched:
        raise ValueError("open faces are built on the uniform column")
    if correction not in CORRECTIONS:
        raise ValueError(f"correction must be one of {CORRECTIONS}, got {correction!r}")
    if normal_halo != "value":
        raise ValueError("normal_halo = :odd is not built (the normal velocity's halo takes the data)")
    if scalar_halo not in ("value", "mirror"):
        raise ValueError("scalar_halo must be 'value' or 'mirror' (the :inflow mode is not built)")
    if outflow != "dirichlet":
        raise ValueError("radiating outflow (:convective, :orlanski) is not built; outflow = 'dirichlet'")
    for need in ("u", "v", "w"):
        if need not in fields:
            raise ValueError("open faces need data for u, v and w")
    hx, hy, hz = grid.halo
    nx, ny, nz = grid.size
    NZ, NY, NX = grid.storage_shape
    x0, y0, z0 = grid.origin
    sides = ([] if x != "open" else ["west", "east"]) + ([] if y != "open" else ["south", "north"])
    planes = []
    for side in sides:
        ax, high = _AXIS[side]
        H, N = grid.halo[ax], grid.size[ax]
        for name in fields:
            if name not in FIELDS:
                raise ValueError(f"unknown open-boundary field {name!r}")
            normal = _NORMAL[name] == ax
            mode = scalar_halo if name == "theta" else "value"
            # _open_range (:46-51): the H halo layers, with the boundary face of
            # the normal component on a low face (interior index 0)
            if high:
                r = np.arange(H + N, N + 2 * H)
            else:
                r = np.arange(0, H + 1 if normal else H)
            st = [_NORMAL[name] == a for a in range(3)]
            xs = np.arange(NX) if ax != 0 else r
            ys = np.arange(NY) if ax != 1 else r
            zs = np.arange(NZ)
            xc = _coord(x0, grid.dx, hx, xs, st[0])
            yc = _coord(y0, grid.dy, hy, ys, st[1])
            zc = _coord(z0, grid.dz, hz, zs, st[2])
            if mode == "mirror":
                vals = np.zeros((len(zs), len(ys), len(xs)))
            else:
                vals = np.array(data.value(name, xc, yc, zc, zs), dtype=np.float64)
            fluid = np.ones((ny if ax == 0 else nx, nz), dtype=bool)
            planes.append(OpenPlane(name, side, ax, high, normal, mode, int(r[0]), np.ascontiguousarray(vals), fluid))
    obs = OpenBoundarySet(grid, planes, correction, x == "open", y == "open")
    obs.correct()
    return obs
