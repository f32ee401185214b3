"""Ghost-cell wall reconstruction on cut-cell surfaces and the cut-cell wall model.

Host set-up (as in the reference, serial loops at geometry time):
`build_ghost_stencils` restates `build_ghost_stencils` / `_interp_weights`
(src/CutCell.jl:996-1172): for every sample point of a field location that
the surface touches -- a non-fluid sample with a fluid neighbour (a ghost
point), or a sample hosted by a cut cell -- the unit normal from the level
set's gradient, the signed wall distance dn = phi/|grad phi|, the foot point
on the true surface, the image point at probe = max(|dn|, probe_factor h_n)
out along the normal, and tri-linear weights at the image point restricted to
fluid donors (renormalised; inverse-distance weights over the nearest fluid
samples of a (2R+1)^3 box when none is left).

Per step (CUDA, include/aeolus_b200_ghost.h): the reconstruction of a
Dirichlet value (`reconstruct_wall_velocity!`, `reconstruct_wall_scalar!`
with wall_value, src/CutCell.jl:1187-1216) or a Neumann flux
(`reconstruct_wall_scalar!` with wall_flux, :1218-1266) into the ghost
points of a storage-layout field on the device, the resolved wall shear
stress nu |u_t(image)| / probe (`wall_shear_stress`, :1268-1336), and the
modelled stress and the slip velocity of a wall law
(src/wall_models/cutcell.jl: `wall_shear_stress(..., law)`,
`wall_slip_velocity`), with the laws of src/wall_models/laws.jl (Spalding,
the rough log law, Monin-Obukhov with the Businger-Dyer-Beljaars-Holtslag
functions).  No CPU fallback: the device calls raise when the library is
missing.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from .cutcell import CutCellGeometry, normal_from

LOCS = {"c": (0, (0.0, 0.0, 0.0)), "fx": (1, (-0.5, 0.0, 0.0)), "fy": (2, (0.0, -0.5, 0.0)),
        "fz": (3, (0.0, 0.0, -0.5))}
_NBR6 = ((1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1))   # (di, dj, dk)


# ----------------------------------------------------------------------------- wall laws
@dataclass
class SpaldingLaw:
    """Spalding's smooth-wall law (src/wall_models/laws.jl:72-106)."""
    kappa: float = 0.41
    B: float = 5.2
    code = 1

    def params(self):
        return (self.kappa, self.B, 0.0, 0.0, 0.0)


LEE_MOSER_2015 = SpaldingLaw(kappa=0.384, B=4.27)


@dataclass
class RoughLogLaw:
    """The neutral log law over a fully rough wall, u_tau = kappa U / ln(h/z0)
    (src/wall_models/laws.jl:207-232; kappa = 0.40, the surface constants')."""
    z0: float
    kappa: float = 0.40
    code = 2

    def params(self):
        return (self.kappa, self.z0, 0.0, 0.0, 0.0)


@dataclass
class MOSTWallLaw:
    """The rough-wall law with the Monin-Obukhov correction for a held
    Obukhov length L (inf: neutral), the Businger-Dyer-Beljaars-Holtslag
    psi_m (src/wall_models/laws.jl:234-284, src/SurfaceExchange.jl:189-225,
    :440), minimum wind U_min."""
    z0m: float
    L: float = math.inf
    U_min: float = 0.1
    kappa: float = 0.40
    code = 3

    def params(self):
        return (self.kappa, self.z0m, self.L, self.U_min, 0.0)


# ----------------------------------------------------------------------------- stencils
def sample_fields(geom: CutCellGeometry, loc: str):
    """`_sample_fields` (src/CutCell.jl:941-982): the level set at the sample
    points of `loc` (the mean of the two cells a face separates; the first
    plane keeps its cell's value) and the fluid samples (fluid side and an
    open control volume / face)."""
    phi = geom.phi
    if loc == "c":
        return phi, (phi > 0) & (geom.vol_frac > 0)
    ax = {"fx": 2, "fy": 1, "fz": 0}[loc]
    s = phi.copy()
    sl_hi = [slice(None)] * 3
    sl_lo = [slice(None)] * 3
    sl_hi[ax] = slice(1, None)
    sl_lo[ax] = slice(None, -1)
    s[tuple(sl_hi)] = 0.5 * (phi[tuple(sl_lo)] + phi[tuple(sl_hi)])
    ap = {"fx": geom.ax, "fy": geom.ay, "fz": geom.az}[loc]
    return s, (s > 0) & (ap > 0)


def _host_cut(geom: CutCellGeometry, loc: str) -> np.ndarray:
    """`_host_cut` (src/CutCell.jl:984-992) of every sample point."""
    cut = geom.is_cut
    if loc == "c":
        return cut.copy()
    out = cut.copy()
    if loc == "fx":
        out[:, :, 1:] |= cut[:, :, :-1]
    elif loc == "fy":
        out[:, 1:, :] |= cut[:, :-1, :]
    else:
        out[1:, :, :] |= cut[:-1, :, :]
    return out


@dataclass
class GhostStencils:
    """The stencils of one field location (storage-shaped sample grid
    (Nz+2Hz, Ny+2Hy, Nx+2Hx)): per point its flat storage index, the signed
    wall distance, probe distance, unit normal, foot and image points, up to
    eight donors (flat index, -1 unused) with weights, and the flags."""
    geom: CutCellGeometry
    loc: str
    k: np.ndarray
    j: np.ndarray
    i: np.ndarray
    target: np.ndarray
    dn: np.ndarray
    probe: np.ndarray
    normal: np.ndarray
    xw: np.ndarray
    ximg: np.ndarray
    donors: np.ndarray
    weights: np.ndarray
    exact: np.ndarray
    ghost: np.ndarray
    valid: np.ndarray

    def __len__(self):
        return len(self.target)


def _sample_coord(grid, loc, i, j, k):
    ox, oy, oz = LOCS[loc][1]
    hx, hy, hz = grid.halo
    x0, y0, z0 = grid.origin
    return (x0 + (i - hx + 0.5 + ox) * grid.dx, y0 + (j - hy + 0.5 + oy) * grid.dy,
            z0 + (k - hz + 0.5 + oz) * grid.dz)


def _interp_weights(fl, grid, loc, X, search_radius):
    """`_interp_weights` (src/CutCell.jl:1084-1172), vectorised over the
    image points X = (x, y, z) arrays; the inverse-distance fallback point
    by point.  Returns donors (n, 8), weights (n, 8), exact, valid."""
    n3, n2, n1 = fl.shape
    ox, oy, oz = LOCS[loc][1]
    hx, hy, hz = grid.halo
    x0, y0, z0 = grid.origin
    xi = (X[0] - x0) / grid.dx + hx - 0.5 - ox
    eta = (X[1] - y0) / grid.dy + hy - 0.5 - oy
    zeta = (X[2] - z0) / grid.dz + hz - 0.5 - oz
    i0 = np.clip(np.floor(xi).astype(np.int64), 0, max(n1 - 2, 0))
    j0 = np.clip(np.floor(eta).astype(np.int64), 0, max(n2 - 2, 0))
    k0 = np.clip(np.floor(zeta).astype(np.int64), 0, max(n3 - 2, 0))
    tx = np.clip(xi - i0, 0.0, 1.0)
    ty = np.clip(eta - j0, 0.0, 1.0)
    tz = np.clip(zeta - k0, 0.0, 1.0)
    n = len(i0)
    donors = np.full((n, 8), -1, dtype=np.int64)
    weights = np.zeros((n, 8))
    wsum = np.zeros(n)
    exact = np.ones(n, dtype=bool)
    m = 0
    for c in (0, 1):
        for b in (0, 1):
            for a in (0, 1):
                w = (1.0 - tx if a == 0 else tx) * (1.0 - ty if b == 0 else ty) * (1.0 - tz if c == 0 else tz)
                ii = np.minimum(i0 + a, n1 - 1)
                jj = np.minimum(j0 + b, n2 - 1)
                kk = np.minimum(k0 + c, n3 - 1)
                f = fl[kk, jj, ii]
                donors[:, m] = np.where(f, (kk * n2 + jj) * n1 + ii, -1)
                weights[:, m] = np.where(f, w, 0.0)
                wsum += np.where(f, w, 0.0)
                exact &= f | ~(w > 0)
                m += 1
    valid = wsum > 1e-12
    weights[valid] /= wsum[valid][:, None]
    for p in np.flatnonzero(~valid):
        # inverse-distance weights over the nearest fluid samples
        best_d = [math.inf] * 8
        best_i = [-1] * 8
        for c in range(-search_radius, search_radius + 1):
            for b in range(-search_radius, search_radius + 1):
                for a in range(-search_radius, search_radius + 1):
                    ii, jj, kk = i0[p] + a, j0[p] + b, k0[p] + c
                    if not (0 <= ii < n1 and 0 <= jj < n2 and 0 <= kk < n3) or not fl[kk, jj, ii]:
                        continue
                    Y = _sample_coord(grid, loc, ii, jj, kk)
                    d2 = (Y[0] - X[0][p]) ** 2 + (Y[1] - X[1][p]) ** 2 + (Y[2] - X[2][p]) ** 2
                    pos = next((q for q in range(8) if d2 < best_d[q]), -1)
                    if pos < 0:
                        continue
                    best_d[pos + 1:] = best_d[pos:7]
                    best_i[pos + 1:] = best_i[pos:7]
                    best_d[pos], best_i[pos] = d2, (kk * n2 + jj) * n1 + ii
        donors[p] = -1
        weights[p] = 0.0
        exact[p] = False
        if best_i[0] < 0:
            continue
        ws = 0.0
        for q in range(8):
            if best_i[q] < 0:
                continue
            w = 1.0 / (best_d[q] + 1e-30)
            donors[p, q], weights[p, q] = best_i[q], w
            ws += w
        weights[p] /= ws
        valid[p] = True
    return donors, weights, exact, valid


def build_ghost_stencils(geom: CutCellGeometry, loc: str = "c", probe_factor: float = 1.0,
                         search_radius: int = 2) -> GhostStencils:
    """`build_ghost_stencils(geom, mesh, loc; probe_factor, search_radius)`
    (src/CutCell.jl:996-1082) on a level-set geometry (`cut_cell_geometry`)."""
    if geom.phi is None:
        raise ValueError("ghost stencils need a level-set geometry (cut_cell_geometry)")
    if loc not in LOCS:
        raise ValueError(f"loc must be one of {list(LOCS)}")
    grid = geom.grid
    sphi, fl = sample_fields(geom, loc)
    n3, n2, n1 = sphi.shape
    hx, hy, hz = grid.halo
    nx, ny, nz = grid.size
    rng = [[hx, hx + nx], [hy, hy + ny], [hz, hz + nz]]   # i, j, k interior ranges
    d = LOCS[loc][0]
    if d > 0:
        rng[d - 1][1] = min(rng[d - 1][1] + 1, (n1, n2, n3)[d - 1])
    sel = np.zeros(sphi.shape, dtype=bool)
    sel[rng[2][0]:rng[2][1], rng[1][0]:rng[1][1], rng[0][0]:rng[0][1]] = True
    touches = np.zeros(sphi.shape, dtype=bool)
    for di, dj, dk in _NBR6:
        src = [slice(None)] * 3
        dst = [slice(None)] * 3
        for ax, dd in ((2, di), (1, dj), (0, dk)):
            if dd > 0:
                dst[ax], src[ax] = slice(None, -1), slice(1, None)
            elif dd < 0:
                dst[ax], src[ax] = slice(1, None), slice(None, -1)
        touches[tuple(dst)] |= fl[tuple(src)]
    hostcut = _host_cut(geom, loc)
    take = sel & np.where(fl, hostcut, touches | hostcut)
    kk, jj, ii = np.nonzero(take)   # storage order: k outer, i inner (the reference's loop order)
    gx, gy, gz, mag = normal_from(sphi, grid, kk, jj, ii)
    dn = sphi[kk, jj, ii] / mag
    X = _sample_coord(grid, loc, ii, jj, kk)
    hn = np.sqrt((gx * grid.dx) ** 2 + (gy * grid.dy) ** 2 + (gz * grid.dz) ** 2)
    probe = np.maximum(np.abs(dn), probe_factor * hn)
    probe = np.where(probe > 0, probe, hn)
    xw = (X[0] - dn * gx, X[1] - dn * gy, X[2] - dn * gz)
    ximg = (xw[0] + probe * gx, xw[1] + probe * gy, xw[2] + probe * gz)
    donors, weights, exact, valid = _interp_weights(fl, grid, loc, ximg, search_radius)
    return GhostStencils(geom, loc, kk, jj, ii, (kk * n2 + jj) * n1 + ii, dn, probe, np.stack([gx, gy, gz], axis=1),
                         np.stack(xw, axis=1), np.stack(ximg, axis=1), donors, weights, exact,
                         ~fl[kk, jj, ii], valid)


# ----------------------------------------------------------------------------- device
_D = C.POINTER(C.c_double)
_I64 = C.POINTER(C.c_int64)
_U8 = C.POINTER(C.c_uint8)


def _pd(a):
    return a.ctypes.data_as(_D)


class DeviceGhost:
    """The stencils of `st` on the device (aeo_ghost_create).  The fields are
    storage-layout arrays (x fastest, halos included); host arrays pass
    through a device copy, device arrays by pointer."""

    def __init__(self, st: GhostStencils, device: int = 0):
        lib = L.load()
        self.st = st
        n3, n2, n1 = st.geom.grid.storage_shape
        self.shape = (n3, n2, n1)
        flags = (st.ghost.astype(np.uint8) | (st.valid.astype(np.uint8) << 1))
        self._keep = [np.ascontiguousarray(st.target, dtype=np.int64),
                      np.ascontiguousarray(st.donors, dtype=np.int64),
                      np.ascontiguousarray(st.weights, dtype=np.float64),
                      np.ascontiguousarray(st.dn, dtype=np.float64),
                      np.ascontiguousarray(st.probe, dtype=np.float64),
                      np.ascontiguousarray(st.normal, dtype=np.float64),
                      np.ascontiguousarray(flags, dtype=np.uint8)]
        t, dnr, w, dn, pr, nrm, fl = self._keep
        h = C.c_void_p()
        L.check(lib.aeo_ghost_create(n1, n2, n3, len(st), t.ctypes.data_as(_I64), dnr.ctypes.data_as(_I64),
                                     _pd(w), _pd(dn), _pd(pr), _pd(nrm), fl.ctypes.data_as(_U8), int(device),
                                     C.byref(h)), None, ghost=True)
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            L.load().aeo_ghost_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def _chk(self, s):
        L.check(s, self._h, ghost=True)

    def reconstruct(self, field: np.ndarray, wall_value=None, wall_flux=None, kappa: float = 1.0) -> np.ndarray:
        """reconstruct_wall_velocity! / reconstruct_wall_scalar! on a host
        storage array (a copy is returned): exactly one of wall_value
        (Dirichlet) and wall_flux (Neumann, kappa d/dn = flux into the fluid)."""
        if (wall_value is None) == (wall_flux is None):
            raise ValueError("give either wall_value (Dirichlet) or wall_flux (Neumann), not both")
        if wall_flux is not None and kappa == 0:
            raise ValueError("kappa must be nonzero for a flux boundary condition")
        f = np.ascontiguousarray(field, dtype=np.float64).copy()
        if f.shape != self.shape:
            raise ValueError(f"field shape {f.shape} != storage shape {self.shape}")
        mode, val = (0, float(wall_value)) if wall_value is not None else (1, float(wall_flux))
        self._chk(L.load().aeo_ghost_reconstruct_host(self._h, _pd(f), mode, val, float(kappa)))
        return f

    def reconstruct_device(self, ptr: int, fp32: bool = False, wall_value=None, wall_flux=None,
                           kappa: float = 1.0, stream: int = 0):
        """The same in place on a device storage array (FP64, or FP32 with fp32)."""
        if (wall_value is None) == (wall_flux is None):
            raise ValueError("give either wall_value (Dirichlet) or wall_flux (Neumann), not both")
        mode, val = (0, float(wall_value)) if wall_value is not None else (1, float(wall_flux))
        self._chk(L.load().aeo_ghost_reconstruct(self._h, C.c_void_p(ptr), 1 if fp32 else 0, mode, val, float(kappa),
                                                 C.c_void_p(stream)))

    def wall_stress(self, u, v, w, nu=None, law=None, nu_eff=None):
        """The wall shear stress at every stencil (CellCenter stencils): the
        resolved nu |u_t(image)|/probe without a law, else the law's u_tau^2,
        and the slip velocity (n, 3) of the law (zero without one); u, v, w
        host storage arrays, the geometry's apertures for the face-to-centre
        average."""
        if self.st.loc != "c":
            raise ValueError("the wall stress takes CellCenter stencils")
        if law is None and nu is None:
            raise ValueError("the resolved stress needs nu")
        if isinstance(law, SpaldingLaw) and nu is None:
            raise ValueError("SpaldingLaw: the kinematic viscosity nu is required")
        if law is not None and nu_eff is None and nu is None:
            raise ValueError("wall_slip_velocity: nu_eff (or nu) is required")
        g = self.st.geom
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (u, v, w, g.ax, g.ay, g.az)]
        for a in arrs:
            if a.shape != self.shape:
                raise ValueError("velocity and aperture arrays must have the storage shape")
        n = len(self.st)
        tau = np.empty(n)
        slip = np.empty((n, 3))
        prm = np.ascontiguousarray(law.params() if law is not None else (0.0,) * 5, dtype=np.float64)
        code = law.code if law is not None else 0
        nuv = float(nu) if nu is not None else float("nan")
        nue = float(nu_eff if nu_eff is not None else (nu if nu is not None else float("nan")))
        self._chk(L.load().aeo_ghost_wall_stress_host(self._h, *[_pd(a) for a in arrs], int(code), _pd(prm), nuv,
                                                      nue, _pd(tau), _pd(slip)))
        return tau, slip
