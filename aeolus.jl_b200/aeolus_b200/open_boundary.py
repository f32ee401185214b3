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
time, :330-380); outflow `:dirichlet` (every point takes the data),
`:convective` or `:orlanski` per side (src/boundary_conditions/outflow.jl: an
outflow point is advanced by the radiation equation with the outward normal
velocity, or the Orlanski phase speed, on the device before every
projection); normal halo `:value`;
scalar halo `:value` or `:mirror`; corrections `:uniform`, `:outflow_only`
and `:none`.  Dirichlet buffers are static, so their correction is applied
once here (the reference applies the same correction to the same data
before every projection); with a radiating face the step redoes data,
radiation and correction before every projection.
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

    def __init__(self, grid: Grid, planes, correction: str, open_x: bool, open_y: bool, outflow=None):
        self.grid = grid
        self.planes = planes
        self.correction = correction
        self.open_x = open_x
        self.open_y = open_y
        self.outflow = dict(outflow or {})          # side -> "dirichlet" | "convective"
        self.ledger = {"Q": 0.0, "residual": 0.0, "delta": 0.0}
        for p in planes:
            p.raw = p.data.copy()                    # the data before the correction

    def mark_solids(self, solid):
        """Where a solid obstacle touches the open faces (`mark_open_boundary_solids!`,
        src/boundary_conditions/open_boundary.jl:809-868): `solid` a storage-shaped
        bool array ([k, j, i], True = solid).  A boundary point is solid when an
        interior cell it borders is (the cell next to the face; for a
        component staggered along the face either of its two cells); solid
        points take zero velocity in every layer (_apply_solid_values!,
        :870-900) and leave the mass-flux correction.  The planes are refilled
        from the data and corrected again."""
        g = self.grid
        solid = np.asarray(solid, dtype=bool)
        if solid.shape != g.storage_shape:
            raise ValueError(f"the solid mask must have the storage shape {g.storage_shape}")
        H = g.halo
        N = g.size
        for p in self.planes:
            ax = p.axis
            t1, t2 = (1, 2) if ax == 0 else (0, 2)
            nl = _NORMAL[p.name]
            cell = H[ax] + N[ax] - 1 if p.high else H[ax]
            fl = np.zeros((N[t1], N[t2]), dtype=bool)
            for da in ((0, -1) if nl == t1 else (0,)):
                for db in ((0, -1) if nl == t2 else (0,)):
                    I = [None, None, None]
                    I[ax] = cell
                    I[t1] = slice(H[t1] + da, H[t1] + N[t1] + da)
                    I[t2] = slice(H[t2] + db, H[t2] + N[t2] + db)
                    fl |= solid[I[2], I[1], I[0]].T          # [tangential, z]
            p.fluid = ~fl
            p.data = p.raw.copy()
        for p in self.planes:
            if p.name == "theta" or p.fluid.all():
                continue
            t1 = 1 if p.axis == 0 else 0
            sol = ~p.fluid                                  # [tangential a, z b]
            for arr in (p.raw, p.data):
                if p.axis == 0:
                    view = arr[H[2]:H[2] + N[2], H[1]:H[1] + N[1], :]      # [k, j, layer]
                    view[sol.T] = 0.0
                else:
                    view = arr[H[2]:H[2] + N[2], :, H[0]:H[0] + N[0]]      # [k, layer, i]
                    view.transpose(0, 2, 1)[sol.T] = 0.0
        self.correct()

    @property
    def radiating(self):
        """The per-side outflow codes (west, east, south, north): 0 :dirichlet,
        1 :convective, 2 :orlanski."""
        code = {"dirichlet": 0, "convective": 1, "orlanski": 2}
        return np.array([code[self.outflow.get(sd, "dirichlet")] for sd in ("west", "east", "south", "north")],
                        dtype=np.int32)

    @property
    def correction_code(self):
        return CORRECTIONS.index(self.correction)

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
        wa = area * self.weight(p).T
        out = s * vals
        q = float(np.sum(np.where(f, out * wa, 0.0)))
        ao = float(np.sum(np.where(f & (out > 0), wa, 0.0)))
        aa = float(np.sum(np.where(f, wa, 0.0)))
        return q, ao, aa

    def weight(self, p):
        """The open fraction of each boundary face of normal plane p ([tangential, z]):
        its aperture when set_apertures gave them, else 1."""
        w = getattr(p, "weight", None)
        return np.ones_like(p.fluid, dtype=np.float64) if w is None else w

    def set_apertures(self, apertures):
        """Weight the mass-flux correction by the open fraction of each boundary
        face (the cut-cell apertures (ax, ay, az) of the projection, face
        layout of aeolus_b200_mgpcg.h), so that the corrected planes carry no
        net flux through the faces the projection sees; a face with aperture
        0 is solid (zero velocity, out of the correction).  The reference's
        correction counts whole faces (`fluid` flags only); with 0/1
        apertures the two agree."""
        g = self.grid
        ax, ay, _ = (np.asarray(a, dtype=np.float64) for a in apertures)
        for p in self.planes:
            if not p.normal:
                continue
            if p.axis == 0:
                w = (ax[:, :, -1] if p.high else ax[:, :, 0]).T        # [j, k]
            else:
                w = (ay[:, -1, :] if p.high else ay[:, 0, :]).T        # [i, k]
            p.weight = np.ascontiguousarray(w)
            p.fluid = p.fluid & (w > 0)
            for arr in (p.raw, p.data):
                H = g.halo
                if p.axis == 0:
                    arr[H[2]:H[2] + g.nz, H[1]:H[1] + g.ny, :][(~p.fluid).T] = 0.0
                else:
                    arr[H[2]:H[2] + g.nz, :, H[0]:H[0] + g.nx].transpose(0, 2, 1)[(~p.fluid).T] = 0.0
        for p in self.planes:
            p.data[...] = p.raw
        self.correct()

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
    def face_weights(self):
        """The weights of the normal planes' boundary faces in the correction
        (0 solid, else the open fraction): x faces [side][Nz][Ny], y faces
        [side][Nz][Nx], FP64."""
        g = self.grid
        xf = np.ones((2, g.nz, g.ny))
        yf = np.ones((2, g.nz, g.nx))
        for p in self.planes:
            if p.normal:
                (xf if p.axis == 0 else yf)[1 if p.high else 0] = (self.weight(p) * p.fluid).T
        return xf, yf

    def packed(self, raw=False):
        """The planes (raw: the data before the correction) as the arrays aeo_set_open takes: x planes
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
            d = p.raw if raw else p.data
            if p.axis == 0:
                xp[f, side, :, :, off:off + n] = d
            else:
                yp[f, side, :, off:off + n, :] = d
        return np.ascontiguousarray(xp), np.ascontiguousarray(yp), modes


def open_boundary_conditions(grid: Grid, data, x: str = "open", y: str = "periodic",
                             fields=FIELDS, correction: str = "uniform", normal_halo: str = "value",
                             scalar_halo: str = "value", outflow: str = "dirichlet", solid=None,
                             apertures=None) -> OpenBoundarySet:
    """A box with open lateral faces fed by `data` (`open_boundary_conditions`,
    :532-638): `x` and `y` each "open" or "periodic" (both faces of an axis
    alike), bottom and top walls.  `fields` names the fields with boundary
    data (the three velocity components and theta); the planes are filled
    from `data` and the normal velocities corrected (`correction`).
    `outflow` is "dirichlet", "convective" or "orlanski", or a dict of those per side;
    `solid` (a storage-shaped bool mask) marks where obstacles touch the
    faces (OpenBoundarySet.mark_solids); `apertures` (the projection's face
    apertures) weight the correction (OpenBoundarySet.set_apertures).
    Raises ValueError for what is not built (an open top or bottom, the
    :odd normal halo, the :inflow scalar halo)."""
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
    sides_all = ("west", "east", "south", "north")
    given_per_side = not isinstance(outflow, str)
    if isinstance(outflow, str):
        outflow = {sd: outflow for sd in sides_all}
    outflow = dict(outflow)
    for sd, mode in outflow.items():
        if sd not in sides_all:
            raise ValueError(f"outflow: unknown side {sd!r} (use {sides_all}; an open top is not built)")
        if mode not in ("dirichlet", "convective", "orlanski"):
            raise ValueError(f"outflow mode must be 'dirichlet', 'convective' or 'orlanski', got {mode!r}")
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
    for sd, mode in outflow.items():
        if mode != "dirichlet" and sd not in sides and given_per_side:
            raise ValueError(f"outflow: side {sd!r} is not an open face of this box")
    obs = OpenBoundarySet(grid, planes, correction, x == "open", y == "open",
                          {sd: outflow.get(sd, "dirichlet") for sd in sides})
    obs.correct()
    if solid is not None:
        obs.mark_solids(solid)
    if apertures is not None:
        obs.set_apertures(apertures)
    return obs
