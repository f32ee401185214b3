"""Reference-state profiles of the sound-proof (anelastic) core.

Restates the profile assembly of `ReferenceState` (src/Anelastic.jl:340-390):
face densities are the logarithmic mean of the neighbouring cells
(`_logmean`, :257-269), the face potential temperature the interpolated
mean, the wall faces take the adjacent cell's value, and every profile gets
its halo-padded twin (`_pad_center`, `_pad_face`, :273-300) so kernels index
it by storage level.

The density profile is prescribed directly, rho(z) = rho0 exp(-z/H) at the
cell centres, rather than integrated hydrostatically from theta; theta_bar
is the initial theta profile (used only by the buoyancy).
"""
from __future__ import annotations

import math

import numpy as np

from .grids import Grid


def logmean(a: float, b: float) -> float:
    """Logarithmic (Lorenz) mean (a-b)/log(a/b) (src/Anelastic.jl:257-269)."""
    if a <= 0 or b <= 0:
        return (a + b) / 2
    s = a + b
    d = a - b
    if d == 0:
        return a
    x = d / s
    if abs(x) < 1e-3:
        x2 = x * x
        return (s / 2) * (1 - x2 / 3 - (4 * x2 * x2) / 45)
    return d / math.log(a / b)


def pad_center(vals: np.ndarray, hz: int) -> np.ndarray:
    """Halo-padded cell profile, extrapolated geometrically (src/Anelastic.jl:273-284)."""
    nz = len(vals)
    out = np.empty(nz + 2 * hz)
    out[hz:hz + nz] = vals
    rb = vals[0] / vals[1] if nz >= 2 else 1.0
    rt = vals[nz - 1] / vals[nz - 2] if nz >= 2 else 1.0
    for h in range(1, hz + 1):
        out[hz - h] = vals[0] * rb ** h
        out[hz + nz - 1 + h] = vals[nz - 1] * rt ** h
    return out


def pad_face(vals: np.ndarray, hz: int, nz: int) -> np.ndarray:
    """Halo-padded face profile (src/Anelastic.jl:286-300), one entry per
    storage face 0 .. Nz+2Hz (the last, above every stencil, extrapolated too)."""
    n = len(vals)
    assert n == nz + 1
    out = np.empty(nz + 2 * hz + 1)
    out[hz:hz + nz + 1] = vals
    rb = vals[0] / vals[1]
    rt = vals[n - 1] / vals[n - 2]
    for h in range(1, hz + 1):
        out[hz - h] = vals[0] * rb ** h
        idx = hz + nz + h
        if idx < len(out):
            out[idx] = vals[n - 1] * rt ** h
    return out


def exponential_density(grid: Grid, rho0: float = 1.2, scale_height: float = 8000.0) -> np.ndarray:
    """rho(z) = rho0 exp(-z/H) at the interior cell centres."""
    return rho0 * np.exp(-grid.znodes("c") / scale_height)


def face_interpolation_weights(grid: Grid):
    """(wlo, whi) of the centre -> face interpolation at interior faces 1..Nz-1
    (src/StretchedGrids.jl:579-581; 1/2 each on a uniform column)."""
    dzc = grid.cell_thickness()
    if grid.zf is None:
        return np.full(grid.nz - 1, 0.5), np.full(grid.nz - 1, 0.5)
    wlo = dzc[1:] / (dzc[:-1] + dzc[1:])
    whi = dzc[:-1] / (dzc[:-1] + dzc[1:])
    return wlo, whi


def anelastic_profiles(grid: Grid, rho_c: np.ndarray, theta_c: np.ndarray) -> dict:
    """The padded weights Wc (Nz+2Hz), Wf (Nz+2Hz+1) and the face reference
    theta (Nz+2Hz+1) the anelastic core needs (src/Anelastic.jl:359-380)."""
    nz, hz = grid.nz, grid.halo[2]
    rho_c = np.asarray(rho_c, dtype=np.float64)
    theta_c = np.asarray(theta_c, dtype=np.float64)
    if rho_c.shape != (nz,) or theta_c.shape != (nz,):
        raise ValueError("profiles must have Nz entries")
    if np.any(rho_c <= 0) or np.any(theta_c <= 0):
        raise ValueError("reference density and potential temperature must be positive")
    wlo, whi = face_interpolation_weights(grid)
    rho_f = np.empty(nz + 1)
    th_f = np.empty(nz + 1)
    rho_f[0] = rho_c[0]
    th_f[0] = theta_c[0]
    for k in range(1, nz):
        rho_f[k] = logmean(rho_c[k - 1], rho_c[k])
        if grid.zf is None:
            th_f[k] = (theta_c[k - 1] + theta_c[k]) / 2
        else:
            th_f[k] = wlo[k - 1] * theta_c[k - 1] + whi[k - 1] * theta_c[k]
    rho_f[nz] = rho_c[nz - 1]
    th_f[nz] = theta_c[nz - 1]
    return {
        "wc": pad_center(rho_c, hz),
        "wf": pad_face(rho_f, hz, nz),
        "thf": pad_face(th_f, hz, nz),
        "rho_c": rho_c,
        "rho_f": rho_f,
        "theta_c": theta_c,
        "theta_f": th_f,
    }
