"""Seeded synthetic inputs of the benchmark cases.

All noise comes from the counter-based Philox4x32-10 generator the reference
uses for reproducible streams (`philox4x32`, `counter_rng`,
src/Backends.jl:1607-1739): key = (seed >> 32, seed), counter =
(block 0, stream, id lo, id hi) with id the interior linear cell index
(x fastest) and stream a field number, and the first 64-bit draw
x1 << 32 | x0 mapped to [0, 1) by its top 53 bits.  The same numbers come
from `aeo_fill_uniform` on the device.
"""
from __future__ import annotations

import numpy as np

from .grids import Grid

_M0 = np.uint64(0xD2511F53)
_M1 = np.uint64(0xCD9E8D57)
_W0 = np.uint32(0x9E3779B9)
_W1 = np.uint32(0xBB67AE85)
_MASK = np.uint64(0xFFFFFFFF)

STREAM_U, STREAM_V, STREAM_W, STREAM_THETA = 0, 1, 2, 3


def philox4x32(ctr, key):
    """Philox4x32-10 block function on arrays (src/Backends.jl:1621-1636).
    ctr: 4 uint32 arrays (or scalars), key: 2 uint32 values."""
    c0, c1, c2, c3 = (np.asarray(c, dtype=np.uint32) for c in ctr)
    k0 = np.uint32(key[0])
    k1 = np.uint32(key[1])
    with np.errstate(over="ignore"):
        for r in range(10):
            p0 = _M0 * c0.astype(np.uint64)
            p1 = _M1 * c2.astype(np.uint64)
            hi0 = (p0 >> np.uint64(32)).astype(np.uint32)
            lo0 = (p0 & _MASK).astype(np.uint32)
            hi1 = (p1 >> np.uint64(32)).astype(np.uint32)
            lo1 = (p1 & _MASK).astype(np.uint32)
            c0, c1, c2, c3 = hi1 ^ c1 ^ k0, lo1, hi0 ^ c3 ^ k1, lo0
            if r < 9:
                k0 = np.uint32((int(k0) + int(_W0)) & 0xFFFFFFFF)
                k1 = np.uint32((int(k1) + int(_W1)) & 0xFFFFFFFF)
    return c0, c1, c2, c3


def philox_uniform(seed: int, stream: int, n: int) -> np.ndarray:
    """U[0, 1) draws of the streams (seed, stream, id) for id in 0..n-1."""
    seed &= (1 << 64) - 1
    ids = np.arange(n, dtype=np.uint64)
    ctr = (np.zeros(n, np.uint32), np.full(n, stream, np.uint32), (ids & _MASK).astype(np.uint32),
           (ids >> np.uint64(32)).astype(np.uint32))
    x0, x1, _, _ = philox4x32(ctr, (seed >> 32, seed & 0xFFFFFFFF))
    x = (x1.astype(np.uint64) << np.uint64(32)) | x0.astype(np.uint64)
    return (x >> np.uint64(11)).astype(np.float64) * (2.0 ** -53)


def uniform_noise(grid: Grid, seed: int, stream: int, amp: float) -> np.ndarray:
    """amp*(2U-1) on the interior, shape (Nz, Ny, Nx)."""
    u = philox_uniform(seed, stream, grid.ncells)
    return (amp * (2.0 * u - 1.0)).reshape(grid.nz, grid.ny, grid.nx)


def embed(grid: Grid, interior: np.ndarray) -> np.ndarray:
    """A storage array (zero halos) holding `interior` (Nz, Ny, Nx)."""
    a = grid.zeros()
    a[grid.interior] = interior
    return a


def taylor_green(grid: Grid, seed: int = 1, amp: float = 1e-3):
    """Taylor-Green vortex u = sin x cos y cos z, v = -cos x sin y cos z, w = 0,
    each at its face position, plus seeded uniform noise of amplitude `amp`
    on u, v, w; theta passive with zero mean (uniform noise, mean removed).
    Returns storage arrays (u, v, w, theta)."""
    xc, yc, zc = grid.xnodes("c"), grid.ynodes("c"), grid.znodes("c")
    xf, yf = grid.xnodes("fx"), grid.ynodes("fy")
    Z, Y, X = np.meshgrid(zc, yc, xf, indexing="ij")
    u = np.sin(X) * np.cos(Y) * np.cos(Z)
    Z, Y, X = np.meshgrid(zc, yf, xc, indexing="ij")
    v = -np.cos(X) * np.sin(Y) * np.cos(Z)
    w = np.zeros((grid.nz, grid.ny, grid.nx))
    if amp != 0:
        u = u + uniform_noise(grid, seed, STREAM_U, amp)
        v = v + uniform_noise(grid, seed, STREAM_V, amp)
        w = w + uniform_noise(grid, seed, STREAM_W, amp)
    th = uniform_noise(grid, seed, STREAM_THETA, 1.0)
    th = th - th.mean()
    return embed(grid, u), embed(grid, v), embed(grid, w), embed(grid, th)


_SM1 = np.uint64(0x9E3779B97F4A7C15)
_SM2 = np.uint64(0xBF58476D1CE4E5B9)
_SM3 = np.uint64(0x94D049BB133111EB)


def _splitmix(x):
    """SplitMix64 (src/operators/spectra.jl:257-262) on uint64 arrays."""
    with np.errstate(over="ignore"):
        x = x + _SM1
        x = (x ^ (x >> np.uint64(30))) * _SM2
        x = (x ^ (x >> np.uint64(27))) * _SM3
        return x ^ (x >> np.uint64(31))


def _mode_key(seed, m1, m2, m3):
    """The counter hash of a mode (src/operators/spectra.jl:263-264); negative
    m wrap as two's complement (m % UInt64)."""
    u = lambda m: np.asarray(m, dtype=np.int64).astype(np.uint64)
    s = _splitmix(np.uint64(seed % (1 << 64)))
    return _splitmix(_splitmix(_splitmix(s ^ u(m1)) ^ u(m2)) ^ u(m3))


def _unit(h):
    return ((h >> np.uint64(11)) + np.uint64(1)).astype(np.float64) * 2.0 ** -53


def _mode_normals(h):
    """Three complex standard normals of mode key h by Box-Muller
    (src/operators/spectra.jl:268-275)."""
    out = []
    with np.errstate(over="ignore"):
        for j in (1, 2, 3):
            a = _splitmix(h + np.uint64(2 * j - 1))
            b = _splitmix(h + np.uint64(2 * j))
            rho = np.sqrt(-2 * np.log(_unit(a)))
            phi = 2 * np.pi * _unit(b)
            out.append((rho * np.cos(phi) + 1j * rho * np.sin(phi)) / np.sqrt(2))
    return out


def passot_pouquet(k, u_rms: float = 1.0, k_peak: float = 4.0):
    """E(k) = 16 sqrt(2/pi) u_rms^2 k^4 / k_p^5 exp(-2 (k/k_p)^2) (src/operators/spectra.jl:248-253)."""
    return 16 * np.sqrt(2 / np.pi) * u_rms ** 2 * k ** 4 / k_peak ** 5 * np.exp(-2 * (k / k_peak) ** 2)


def isotropic_turbulence(grid: Grid, u_rms: float = 1.0, k_peak: float = 4.0, seed: int = 1, kmax: float = np.inf):
    """`isotropic_turbulence_field!` (src/operators/spectra.jl:312-343): the
    random-phase solenoidal field of spectrum E(k), defined in spectral space
    (each mode's draw depends on seed and the integer mode only), evaluated
    at each component's staggered nodes.  Triply periodic uniform grids.
    Returns storage arrays (u, v, w)."""
    nx, ny, nz = grid.size
    lx, ly, lz = grid.extent
    mx = np.fft.fftfreq(nx, 1.0 / nx).astype(np.int64)
    my = np.fft.fftfreq(ny, 1.0 / ny).astype(np.int64)
    mz = np.fft.fftfreq(nz, 1.0 / nz).astype(np.int64)
    M3, M2, M1 = np.meshgrid(mz, my, mx, indexing="ij")
    ck = (2 * np.pi / lx, 2 * np.pi / ly, 2 * np.pi / lz)
    dV = ck[0] * ck[1] * ck[2]
    keep = (2 * np.abs(M1) < nx) & (2 * np.abs(M2) < ny) & (2 * np.abs(M3) < nz) & ~((M1 == 0) & (M2 == 0) & (M3 == 0))
    k1, k2, k3 = ck[0] * M1, ck[1] * M2, ck[2] * M3
    kk2 = k1 ** 2 + k2 ** 2 + k3 ** 2
    kk = np.sqrt(kk2)
    keep &= kk <= kmax
    canon = (M3 > 0) | ((M3 == 0) & ((M2 > 0) | ((M2 == 0) & (M1 > 0))))
    sgn = np.where(canon, 1, -1)
    r = _mode_normals(_mode_key(seed, sgn * M1, sgn * M2, sgn * M3))
    kc = (sgn * k1, sgn * k2, sgn * k3)
    safe = np.where(keep, kk2, 1.0)
    kr = (kc[0] * r[0] + kc[1] * r[1] + kc[2] * r[2]) / safe
    amp = np.sqrt(np.maximum(passot_pouquet(kk, u_rms, k_peak), 0.0) * dV / (4 * np.pi * safe))
    x0, y0, z0 = grid.origin
    firsts = ((x0, y0 + 0.5 * grid.dy, z0 + 0.5 * grid.dz), (x0 + 0.5 * grid.dx, y0, z0 + 0.5 * grid.dz),
              (x0 + 0.5 * grid.dx, y0 + 0.5 * grid.dy, z0))
    out = []
    for j in range(3):
        pj = r[j] - kc[j] * kr
        uh = amp * np.where(canon, pj, np.conj(pj))
        x1 = firsts[j]
        A = np.where(keep, uh * np.exp(1j * (k1 * x1[0] + k2 * x1[1] + k3 * x1[2])), 0.0) * (nx * ny * nz)
        out.append(embed(grid, np.real(np.fft.ifftn(A))))
    return tuple(out)


def cbl_theta_profile(z: np.ndarray, theta_ml: float = 300.0, z_inv: float = 1000.0, jump: float = 3.0,
                      lapse: float = 3e-3) -> np.ndarray:
    """Dry convective boundary layer: theta_ml up to z_inv, then a jump and a
    constant lapse rate above."""
    z = np.asarray(z, dtype=np.float64)
    return np.where(z < z_inv, theta_ml, theta_ml + jump + lapse * (z - z_inv))


def cbl_initial(grid: Grid, seed: int = 1, noise: float = 0.1, noise_levels: int = 10):
    """Rest state with the CBL theta profile and seeded uniform +-noise in the
    lowest `noise_levels` levels.  Returns (u, v, w, theta) storage arrays and
    the interior theta profile."""
    prof = cbl_theta_profile(grid.znodes("c"))
    th = np.broadcast_to(prof[:, None, None], (grid.nz, grid.ny, grid.nx)).copy()
    nz_noise = min(noise_levels, grid.nz)
    pert = uniform_noise(grid, seed, STREAM_THETA, noise)
    th[:nz_noise] += pert[:nz_noise]
    z = np.zeros((grid.nz, grid.ny, grid.nx))
    return embed(grid, z), embed(grid, z), embed(grid, z), embed(grid, th), prof


def storage_from_interior(grid: Grid, interior: np.ndarray, wall_face: bool = False) -> np.ndarray:
    """A storage array from its interior values with the halos filled:
    periodic in x and y; in z periodic, or at walls the mirror (zero
    gradient), or for a z-face field zero on the two wall faces and zero
    beyond them."""
    hx, hy, hz = grid.halo
    a = np.pad(interior, ((0, 0), (hy, hy), (hx, hx)), mode="wrap")
    if grid.bc_z == "periodic":
        a = np.pad(a, ((hz, hz), (0, 0), (0, 0)), mode="wrap")
    elif wall_face:
        a = np.pad(a, ((hz, hz), (0, 0), (0, 0)), mode="constant")
        a[hz] = 0.0
        a[hz + grid.nz] = 0.0
    else:
        a = np.pad(a, ((hz, hz), (0, 0), (0, 0)), mode="symmetric")
    return np.ascontiguousarray(a)


def tracer_case(grid: Grid, seed: int, cfl: float = 0.9, sharp: bool = True):
    """Inputs of the positivity-preserving advection: seeded normal face
    velocities scaled so that sum_d max|u_d| dt/dx_d = cfl at dt = 1, and a
    non-negative field -- a smooth positive background with, when sharp,
    random zero cells, a zero slab and a unit block (where the limiter acts).
    Returns storage arrays u, v, w, phi (halos filled) and dt."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = grid.size
    vel = [rng.standard_normal((nz, ny, nx)) for _ in range(3)]
    rate = sum(np.abs(a).max() / h for a, h in zip(vel, (grid.dx, grid.dy, grid.dz)))
    vel = [a * (cfl / rate) for a in vel]
    x = (np.arange(nx) + 0.5) / nx
    y = (np.arange(ny) + 0.5) / ny
    z = (np.arange(nz) + 0.5) / nz
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    phi = 1.5 + np.sin(2 * np.pi * X) * np.cos(2 * np.pi * Y) * np.cos(2 * np.pi * Z)
    if sharp:
        phi = np.where(rng.random((nz, ny, nx)) < 0.15, 0.0, phi)
        phi[nz // 4:nz // 2, ny // 4:ny // 2, nx // 4:nx // 2] = 1.0
        phi[:, :, :nx // 8] = 0.0
    return (storage_from_interior(grid, vel[0]), storage_from_interior(grid, vel[1]),
            storage_from_interior(grid, vel[2], wall_face=True), storage_from_interior(grid, phi), 1.0)
