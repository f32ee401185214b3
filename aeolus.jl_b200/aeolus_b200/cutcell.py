"""Cut-cell geometry of floor-standing box obstacles and the host side of
the cut-cell projection (set-up work: serial loops in the reference too).

Restates `cut_cell_geometry(mesh, levelset; nsub, vol_min)` and
`_finalize_geometry` (src/CutCell.jl:243-319, :398-493):
  * volume fractions from nsub^3 sub-samples per cell, open-area fractions
    from nsub^2 samples per face, with the level-set convention phi > 0
    fluid (src/CutCell.jl:265-317);
  * the consistency sweeps: a face touching a dry cell is closed; a wetted
    cell with no open face becomes solid; repeated up to 16 times until
    nothing changes (:413-447);
  * vol_eff = max(vol_frac, vol_min) on wetted cells, 0 in solid (:449-465).
The outermost low-side storage faces are closed as in the reference (:407-411).

Obstacles are axis-aligned boxes standing on the floor z0 (an urban block
model).  Their union with the ground is the level set
phi(x, y, z) = z - H(x, y), H the top of the tallest box whose closed
footprint covers (x, y) (the floor elsewhere), periodic in x and y: a sample
is fluid iff it lies strictly above H.  The per-sample test is done as a
sorted search of the z samples, so the fractions are the reference's exact
sample counts at any grid size.

Arrays are storage-shaped (Nz+2Hz, Ny+2Hy, Nx+2Hx) and indexed [k, j, i];
ax[k, j, i] is the west face of cell i, ay the south face, az the bottom.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Callable, Optional

import numpy as np

from .grids import Grid
from .inputs import philox_uniform, uniform_noise


@dataclass
class CutCellGeometry:
    grid: Grid
    vol_frac: np.ndarray
    vol_eff: np.ndarray
    ax: np.ndarray
    ay: np.ndarray
    az: np.ndarray
    is_solid: np.ndarray
    is_small: np.ndarray
    vol_min: float
    nsub: int
    # the small cells' merge partners (flat storage index, -1 none), the cut
    # cells, and from a level set its cell-centre values, the unit normals
    # into the fluid and the wetted area of every cut cell
    merge_target: Optional[np.ndarray] = None
    is_cut: Optional[np.ndarray] = None
    phi: Optional[np.ndarray] = None
    nx: Optional[np.ndarray] = None
    ny: Optional[np.ndarray] = None
    nz: Optional[np.ndarray] = None
    area: Optional[np.ndarray] = None

    @property
    def fluid_interior(self) -> np.ndarray:
        return ~self.is_solid[self.grid.interior]


def random_boxes(grid: Grid, n: int, seed: int, footprint=(10.0, 40.0), height=(10.0, 60.0)) -> np.ndarray:
    """n floor-standing boxes: Philox-seeded centres uniform over the
    horizontal domain, side lengths uniform in `footprint`, heights uniform in
    `height`.  Returns (n, 6) rows (x0, x1, y0, y1, z0, z1)."""
    u = [philox_uniform(seed, 100 + s, n) for s in range(5)]
    lx, ly = grid.extent[0], grid.extent[1]
    ox, oy, oz = grid.origin
    cx, cy = ox + u[0] * lx, oy + u[1] * ly
    wx = footprint[0] + u[2] * (footprint[1] - footprint[0])
    wy = footprint[0] + u[3] * (footprint[1] - footprint[0])
    hz = height[0] + u[4] * (height[1] - height[0])
    return np.stack([cx - wx / 2, cx + wx / 2, cy - wy / 2, cy + wy / 2, np.full(n, oz), oz + hz], axis=1)


def _west(grid: Grid, axis: int) -> np.ndarray:
    """_xw/_yw/_zw of every storage index (src/CutCell.jl:90-92)."""
    n, H = grid.size[axis], grid.halo[axis]
    d = (grid.dx, grid.dy, grid.dz)[axis]
    return grid.origin[axis] + (np.arange(n + 2 * H) - H) * d


def _subsamples(grid: Grid, axis: int, nsub: int) -> np.ndarray:
    """x_w + (a - 1/2) h, h = d/nsub, a = 1..nsub, for every storage index,
    flattened cell-major (src/CutCell.jl:266-274)."""
    d = (grid.dx, grid.dy, grid.dz)[axis]
    h = d * (1.0 / nsub)
    return (_west(grid, axis)[:, None] + (np.arange(1, nsub + 1) - 0.5) * h).ravel()


def box_heights(grid: Grid, boxes, x: np.ndarray, y: np.ndarray) -> np.ndarray:
    """H on the lattice y (rows) x x (columns): the tallest box whose closed
    footprint holds the point, periodic in x and y; the floor z0 elsewhere."""
    lx, ly = grid.extent[0], grid.extent[1]
    ox, oy, floor = grid.origin
    X = ox + np.mod(x - ox, lx)
    Y = oy + np.mod(y - oy, ly)
    H = np.full((len(Y), len(X)), floor)
    for (x0, x1, y0, y1, z0, z1) in np.asarray(boxes, dtype=np.float64).reshape(-1, 6):
        if z0 > floor:
            raise ValueError("boxes must stand on the floor (z0 <= grid origin z)")
        for sx in (-lx, 0.0, lx):
            ix = np.nonzero((X >= x0 + sx) & (X <= x1 + sx))[0]
            if ix.size == 0:
                continue
            for sy in (-ly, 0.0, ly):
                iy = np.nonzero((Y >= y0 + sy) & (Y <= y1 + sy))[0]
                if iy.size == 0:
                    continue
                H[np.ix_(iy, ix)] = np.maximum(H[np.ix_(iy, ix)], z1)
    return H


def _level_fractions(nle: np.ndarray, nsub: int, nz: int, fold, norm: float) -> np.ndarray:
    """Fluid fraction of every level from nle, the number of z samples at or
    below H of each sample column: level k owns samples [k nsub, (k+1) nsub),
    and fold sums a level's per-column counts over the samples of each cell
    or face.  Levels above the tallest H are all fluid, so only the levels
    the obstacles reach are counted (one level at a time)."""
    top = min(nz, int(nle.max()) // nsub + 1)
    first = fold(nsub - np.clip(nle, 0, nsub))
    out = np.ones((nz,) + first.shape)
    out[0] = first / norm
    for k in range(1, top):
        out[k] = fold(nsub - np.clip(nle - k * nsub, 0, nsub)) / norm
    return out


def box_geometry(grid: Grid, boxes, nsub: int = 4, vol_min: float = 1e-3) -> CutCellGeometry:
    """`cut_cell_geometry` of floor-standing boxes (src/CutCell.jl:243-319)."""
    if nsub < 1:
        raise ValueError("nsub must be >= 1")
    if not 0 <= vol_min < 1:
        raise ValueError("vol_min must lie in [0, 1)")
    NZ, NY, NX = grid.storage_shape
    xs, ys, zs = (_subsamples(grid, a, nsub) for a in range(3))
    xf, yf, zf = (_west(grid, a) for a in range(3))
    n2, n3 = float(nsub * nsub), float(nsub ** 3)
    Hc = box_heights(grid, boxes, xs, ys)

    def below(H):
        return np.searchsorted(zs, H, side="right")    # samples with z <= H

    vol = _level_fractions(below(Hc), nsub, NZ, lambda c: c.reshape(NY, nsub, NX, nsub).sum(axis=(1, 3)), n3)
    ax = _level_fractions(below(box_heights(grid, boxes, xf, ys)), nsub, NZ,
                          lambda c: c.reshape(NY, nsub, NX).sum(axis=1), n2)
    ay = _level_fractions(below(box_heights(grid, boxes, xs, yf)), nsub, NZ,
                          lambda c: c.reshape(NY, NX, nsub).sum(axis=2), n2)
    nle = np.searchsorted(zf, Hc, side="right")       # bottom faces with z <= H
    az = np.ones((NZ, NY, NX))
    for k in range(min(NZ, int(nle.max()) + 1)):
        az[k] = (nle <= k).reshape(NY, nsub, NX, nsub).sum(axis=(1, 3)) / n2
    return finalize_geometry(grid, vol, ax, ay, az, vol_min, nsub)


def box_solid_mask(grid: Grid, boxes) -> np.ndarray:
    """The SolidMask of floor-standing boxes: a cell is solid when its centre
    lies below the top of a box whose closed footprint holds it (the
    predicate of mark_solid!, src/IBM.jl:51-63), evaluated on every storage
    cell, so the x and y halos hold the periodic images and the levels below
    the floor are solid (mark_solid! marks the interior only; the halo cells
    only decide the faces on the domain boundary, which are periodic partners
    or walls)."""
    xc, yc = (_subsamples(grid, a, 1) for a in range(2))
    H = box_heights(grid, boxes, xc, yc)
    return storage_zc(grid)[:, None, None] < H[None, :, :]


def storage_zc(grid: Grid) -> np.ndarray:
    """Cell-centre heights of every storage level: uniform, or on a stretched
    column from its faces, the halo faces continued linearly (the halo
    levels mirror the first and last cells, src/StretchedGrids.jl:345-360)."""
    if grid.zf is None:
        return _subsamples(grid, 2, 1)
    H, nz = grid.halo[2], grid.nz
    zf = np.empty(nz + 2 * H + 1)
    zf[H:H + nz + 1] = grid.zf
    for k in range(H - 1, -1, -1):
        zf[k] = 2 * zf[k + 1] - zf[k + 2]
    for k in range(H + nz + 1, nz + 2 * H + 1):
        zf[k] = 2 * zf[k - 1] - zf[k - 2]
    return 0.5 * (zf[:-1] + zf[1:])


def staircase_geometry(grid: Grid, mask: np.ndarray, vol_min: float = 1e-3) -> CutCellGeometry:
    """`cut_cell_geometry(mesh, sm::SolidMask)` (src/CutCell.jl:334-352): 0/1
    volume fractions and apertures (a face is open when both its cells are
    fluid), then the consistency passes, so the cut-cell operators are the
    Cartesian ones with blocked faces.  This is the obstacle model of the
    urban cases (their `geom.sm` solid mask)."""
    mask = np.asarray(mask, dtype=bool)
    if mask.shape != grid.storage_shape:
        raise ValueError(f"mask shape {mask.shape} != storage shape {grid.storage_shape}")
    vol = np.where(mask, 0.0, 1.0)
    fl = ~mask
    ax = np.zeros(grid.storage_shape)
    ay = np.zeros(grid.storage_shape)
    az = np.zeros(grid.storage_shape)
    ax[:, :, 1:] = fl[:, :, :-1] & fl[:, :, 1:]
    ay[:, 1:, :] = fl[:, :-1, :] & fl[:, 1:, :]
    az[1:, :, :] = fl[:-1, :, :] & fl[1:, :, :]
    return finalize_geometry(grid, vol, ax, ay, az, vol_min, 1)


def _storage_coord(grid: Grid, axis: int, face: bool) -> np.ndarray:
    """Cell-centre (face=False) or west-face coordinate of every storage index
    along `axis` of a uniform grid (_xc/_xw, src/CutCell.jl:90-92)."""
    n, H = grid.size[axis], grid.halo[axis]
    d = (grid.dx, grid.dy, grid.dz)[axis]
    return grid.origin[axis] + (np.arange(n + 2 * H) - H + (0.0 if face else 0.5)) * d


def cut_cell_geometry(grid: Grid, levelset: Callable, nsub: int = 4, vol_min: float = 1e-3) -> CutCellGeometry:
    """`cut_cell_geometry(mesh, levelset; nsub, vol_min)` (src/CutCell.jl:243-319)
    for a level set phi(x, y, z) (phi > 0 fluid) that takes numpy arrays:
    phi at every storage cell centre, volume fractions from nsub^3 sub-samples
    per cell and open-area fractions from nsub^2 per face, then the
    robustness passes, the small-cell merge partners, the normals and the
    wetted areas (_finalize_geometry)."""
    if grid.zf is not None:
        raise ValueError("cut_cell_geometry takes a uniform (RegularGrid) column")
    if nsub < 1:
        raise ValueError("nsub must be >= 1")
    if not 0 <= vol_min < 1:
        raise ValueError("vol_min must lie in [0, 1)")
    xc, yc, zc = (_storage_coord(grid, a, False) for a in range(3))
    xw, yw, zw = (_storage_coord(grid, a, True) for a in range(3))
    h = (grid.dx / nsub, grid.dy / nsub, grid.dz / nsub)
    off = (np.arange(nsub) + 0.5)

    def ls(x, y, z):
        return np.asarray(levelset(x[None, None, :], y[None, :, None], z[:, None, None]), dtype=np.float64) * \
            np.ones((len(z), len(y), len(x)))

    phi = ls(xc, yc, zc)
    vol = np.zeros(phi.shape)
    for c in off:
        for b in off:
            for a in off:
                vol += ls(xw + a * h[0], yw + b * h[1], zw + c * h[2]) > 0
    vol /= nsub ** 3
    ax = np.zeros(phi.shape)
    ay = np.zeros(phi.shape)
    az = np.zeros(phi.shape)
    for c in off:
        for b in off:
            ax += ls(xw, yw + b * h[1], zw + c * h[2]) > 0
    for c in off:
        for a in off:
            ay += ls(xw + a * h[0], yw, zw + c * h[2]) > 0
    for b in off:
        for a in off:
            az += ls(xw + a * h[0], yw + b * h[1], zw) > 0
    ax /= nsub ** 2
    ay /= nsub ** 2
    az /= nsub ** 2
    return finalize_geometry(grid, vol, ax, ay, az, vol_min, nsub, phi=phi)


def normal_from(phi: np.ndarray, grid: Grid, k, j, i):
    """`_normal_from` (src/CutCell.jl:126-139): the unit normal into the fluid
    from central differences of phi (one-sided at the array edges) and
    |grad phi|; (0, 0, 1, 1) where the gradient vanishes.  Vectorised over
    index arrays k, j, i."""
    n3, n2, n1 = phi.shape
    k, j, i = (np.asarray(a) for a in (k, j, i))
    ip, im = np.minimum(i + 1, n1 - 1), np.maximum(i - 1, 0)
    jp, jm = np.minimum(j + 1, n2 - 1), np.maximum(j - 1, 0)
    kp, km = np.minimum(k + 1, n3 - 1), np.maximum(k - 1, 0)
    with np.errstate(invalid="ignore", divide="ignore"):
        gx = np.where(ip == im, 0.0, (phi[k, j, ip] - phi[k, j, im]) / ((ip - im) * grid.dx))
        gy = np.where(jp == jm, 0.0, (phi[k, jp, i] - phi[k, jm, i]) / ((jp - jm) * grid.dy))
        gz = np.where(kp == km, 0.0, (phi[kp, j, i] - phi[km, j, i]) / ((kp - km) * grid.dz))
        mag = np.sqrt(gx * gx + gy * gy + gz * gz)
        bad = ~(mag > 0) | ~np.isfinite(mag)
        safe = np.where(bad, 1.0, mag)
        return (np.where(bad, 0.0, gx / safe), np.where(bad, 0.0, gy / safe), np.where(bad, 1.0, gz / safe),
                np.where(bad, 1.0, mag))


def finalize_geometry(grid: Grid, vol, ax, ay, az, vol_min: float, nsub: int, phi=None) -> CutCellGeometry:
    """The robustness passes of `_finalize_geometry` (src/CutCell.jl:398-465),
    the merge partner of every small cell (the open neighbour of largest
    volume fraction, the first in the order -x, +x, -y, +y, -z, +z on a tie;
    :467-491) and, with a level set, the wetted area from the aperture
    balance and the normal of every cut cell (:493-504)."""
    vol = np.array(vol, dtype=np.float64)
    ax, ay, az = (np.array(a, dtype=np.float64) for a in (ax, ay, az))
    solid = ~(vol > 0)
    ax[:, :, 0] = 0.0
    ay[:, 0, :] = 0.0
    az[0, :, :] = 0.0
    for _ in range(16):
        ax[:, :, 1:][solid[:, :, :-1] | solid[:, :, 1:]] = 0.0
        ay[:, 1:, :][solid[:, :-1, :] | solid[:, 1:, :]] = 0.0
        az[1:, :, :][solid[:-1, :, :] | solid[1:, :, :]] = 0.0
        opn = ax + ay + az
        opn[:, :, :-1] += ax[:, :, 1:]
        opn[:, :-1, :] += ay[:, 1:, :]
        opn[:-1, :, :] += az[1:, :, :]
        newly = ~solid & ~(opn > 0)
        if not newly.any():
            break
        solid |= newly
        vol[newly] = 0.0
    small = ~solid & (vol < vol_min)
    cut = ~solid & (vol < 1.0)
    vol_eff = np.where(solid, 0.0, np.where(vol < vol_min, vol_min, vol))
    n3, n2, n1 = vol.shape
    target = np.full(vol.shape, -1, dtype=np.int64)
    for k, j, i in zip(*np.nonzero(small)):
        best, bestv = -1, 0.0
        for ap, i2, j2, k2 in ((ax[k, j, i] if i > 0 else 0.0, i - 1, j, k),
                               (ax[k, j, i + 1] if i < n1 - 1 else 0.0, i + 1, j, k),
                               (ay[k, j, i] if j > 0 else 0.0, i, j - 1, k),
                               (ay[k, j + 1, i] if j < n2 - 1 else 0.0, i, j + 1, k),
                               (az[k, j, i] if k > 0 else 0.0, i, j, k - 1),
                               (az[k + 1, j, i] if k < n3 - 1 else 0.0, i, j, k + 1)):
            if not ap > 0 or not (0 <= i2 < n1 and 0 <= j2 < n2 and 0 <= k2 < n3):
                continue
            if vol[k2, j2, i2] > bestv:
                bestv, best = vol[k2, j2, i2], (k2 * n2 + j2) * n1 + i2
        target[k, j, i] = best
    geom = CutCellGeometry(grid, vol, vol_eff, ax, ay, az, solid, small, vol_min, nsub,
                           merge_target=target, is_cut=cut)
    if phi is not None:
        axp = np.zeros(vol.shape); axp[:, :, :-1] = ax[:, :, 1:]
        ayp = np.zeros(vol.shape); ayp[:, :-1, :] = ay[:, 1:, :]
        azp = np.zeros(vol.shape); azp[:-1, :, :] = az[1:, :, :]
        sx = (axp - ax) * (grid.dy * grid.dz)
        sy = (ayp - ay) * (grid.dx * grid.dz)
        sz = (azp - az) * (grid.dx * grid.dy)
        geom.area = np.where(cut, np.sqrt(sx * sx + sy * sy + sz * sz), 0.0)
        geom.phi = np.asarray(phi, dtype=np.float64)
        geom.nx, geom.ny, geom.nz = np.zeros(vol.shape), np.zeros(vol.shape), np.zeros(vol.shape)
        kk, jj, ii = np.nonzero(cut)
        gx, gy, gz, _ = normal_from(geom.phi, grid, kk, jj, ii)
        geom.nx[cut], geom.ny[cut], geom.nz[cut] = gx, gy, gz
    return geom


def face_coefficients(geom: CutCellGeometry, power: int = 2):
    """Interior face coefficients a^q of the cut-cell Laplacian
    (cutcell_laplacian!, src/CutCell.jl:735-768): cx (Nz, Ny, Nx+1),
    cy (Nz, Ny+1, Nx), cz (Nz+1, Ny, Nx); face index i is the west face of
    cell i, the last one the east face of the last cell."""
    g = geom.grid
    hx, hy, hz = g.halo
    nx, ny, nz = g.size
    ks, js, is_ = slice(hz, hz + nz), slice(hy, hy + ny), slice(hx, hx + nx)
    cx = geom.ax[ks, js, hx:hx + nx + 1] ** power
    cy = geom.ay[ks, hy:hy + ny + 1, is_] ** power
    cz = geom.az[hz:hz + nz + 1, js, is_] ** power
    return np.ascontiguousarray(cx), np.ascontiguousarray(cy), np.ascontiguousarray(cz)


def cutcell_divergence(geom: CutCellGeometry, u, v, w, redistribute: bool = False) -> np.ndarray:
    """`cutcell_divergence!` (src/CutCell.jl:602-622): the aperture-weighted
    flux difference over vol_eff, zero in solid cells; u, v, w storage arrays
    with filled halos.  With `redistribute`, `_redistribute_small_cells!`
    (:624-644): every small cell and its merge partner take their cluster's
    volume-weighted mean, one small cell after another in storage order (a
    partner shared by several small cells accumulates them in turn), which
    conserves the sum of vol_eff times the divergence.  Returns the interior
    (Nz, Ny, Nx)."""
    g = geom.grid
    hx, hy, hz = g.halo
    nx, ny, nz = g.size
    K, J, I = slice(hz, hz + nz), slice(hy, hy + ny), slice(hx, hx + nx)
    Ip, Jp, Kp = slice(hx + 1, hx + nx + 1), slice(hy + 1, hy + ny + 1), slice(hz + 1, hz + nz + 1)
    fx = (geom.ax[K, J, Ip] * u[K, J, Ip] - geom.ax[K, J, I] * u[K, J, I]) / g.dx
    fy = (geom.ay[K, Jp, I] * v[K, Jp, I] - geom.ay[K, J, I] * v[K, J, I]) / g.dy
    fz = (geom.az[Kp, J, I] * w[Kp, J, I] - geom.az[K, J, I] * w[K, J, I]) / g.dz
    ve = geom.vol_eff[K, J, I]
    div = np.where(ve > 0, (fx + fy + fz) / np.where(ve > 0, ve, 1.0), 0.0)
    if not redistribute or geom.merge_target is None or not geom.is_small[K, J, I].any():
        return div
    full = np.zeros(geom.vol_eff.shape)
    full[K, J, I] = div
    flat, vef = full.ravel(), geom.vol_eff.ravel()
    inside = np.zeros(full.shape, dtype=bool)
    inside[K, J, I] = True
    for q in np.flatnonzero((geom.is_small & inside).ravel()):
        t = geom.merge_target.ravel()[q]
        if t < 0:
            continue
        vt = vef[q] + vef[t]
        if not vt > 0:
            continue
        d = (vef[q] * flat[q] + vef[t] * flat[t]) / vt
        flat[q] = d
        flat[t] = d
    return full[K, J, I]


def pressure_rhs(geom: CutCellGeometry, u, v, w) -> np.ndarray:
    """Right-hand side of the symmetric cut-cell projection: vol_eff times
    the cut-cell divergence (vol_eff L is symmetric, src/CutCell.jl:705-716),
    zero in the solid, zero mean over the fluid."""
    g = geom.grid
    ve = geom.vol_eff[g.interior]
    b = ve * cutcell_divergence(geom, u, v, w)
    fluid = ve > 0
    b[fluid] -= b[fluid].mean()
    b[~fluid] = 0.0
    return b


def _periodic_xy(grid: Grid, A: np.ndarray) -> None:
    hx, hy, _ = grid.halo
    nx, ny, _ = grid.size
    A[:, :, :hx] = A[:, :, nx:nx + hx]
    A[:, :, hx + nx:] = A[:, :, hx:2 * hx]
    A[:, :hy, :] = A[:, ny:ny + hy, :]
    A[:, hy + ny:, :] = A[:, hy:2 * hy, :]


def urban_velocity(grid: Grid, geom: CutCellGeometry, u_ref: float = 5.0, z_ref: float = 10.0,
                   z0: float = 0.1, noise: float = 0.5, seed: int = 1):
    """Log-profile inflow u(z) = u_ref ln(z/z0)/ln(z_ref/z0) (zero below z0)
    plus Philox-seeded uniform noise of amplitude `noise` on u, v, w, with
    every closed face zeroed.  Storage arrays with periodic x/y halos and
    zero z halos."""
    z = grid.znodes("c")
    prof = np.where(z > z0, np.log(np.maximum(z, z0) / z0) / np.log(z_ref / z0), 0.0) * u_ref
    comps = (prof[:, None, None] + uniform_noise(grid, seed, 0, noise),
             uniform_noise(grid, seed, 1, noise), uniform_noise(grid, seed, 2, noise))
    out = []
    for a, ap in zip(comps, (geom.ax, geom.ay, geom.az)):
        A = grid.zeros()
        A[grid.interior] = a * (ap[grid.interior] > 0)
        _periodic_xy(grid, A)
        out.append(A)
    return tuple(out)
