"""TEST INFRASTRUCTURE ONLY: a numpy/Python restatement of the ghost-cell wall
reconstruction, the wall shear stress and the wall laws, the checker of
the library's aeo_ghost_* kernels (tests only; the product never imports it).

Follows, line for line in arithmetic order:
  _image_value, _reconstruct_dirichlet!, reconstruct_wall_scalar!  src/CutCell.jl:1174-1266
  wall_shear_stress, _center_velocity                              src/CutCell.jl:1268-1380
  wall_shear_stress(..., law), _each_tangential, wall_slip_velocity
                                                                   src/wall_models/cutcell.jl:48-120
  _exp_tail, spalding_yplus, _increasing_root, friction_velocity   src/wall_models/laws.jl:108-284
  psi_m of BusingerDyerBeljaarsHoltslag, _Phi_m                    src/SurfaceExchange.jl:189-225, :440
The stencils are the host set-up of aeolus_b200.ghost (build_ghost_stencils).
"""
from __future__ import annotations

import math

import numpy as np

EPS = np.finfo(np.float64).eps


def image_value(flat, donors, weights):
    acc = 0.0
    for m in range(8):
        d = donors[m]
        if d < 0:
            continue
        acc += weights[m] * flat[d]
    return acc


def reconstruct(field, st, wall_value=None, wall_flux=None, kappa=1.0):
    """reconstruct_wall_velocity! / reconstruct_wall_scalar! on a copy."""
    f = np.array(field, dtype=np.float64)
    flat = f.ravel()
    for s in range(len(st)):
        if not (st.ghost[s] and st.valid[s]):
            continue
        img = image_value(flat, st.donors[s], st.weights[s])
        if wall_value is not None:
            flat[st.target[s]] = wall_value + (st.dn[s] / st.probe[s]) * (img - wall_value)
        else:
            g = wall_flux * (1.0 / kappa)
            flat[st.target[s]] = img + (st.dn[s] - st.probe[s]) * g
    return f


def center_velocity(u, v, w, geom):
    """_center_velocity: the aperture-weighted mean of each cell's two faces."""
    n3, n2, n1 = u.shape
    out = []
    for f, a, ax in ((u, geom.ax, 2), (v, geom.ay, 1), (w, geom.az, 0)):
        a2 = np.zeros(a.shape)
        f2 = np.zeros(f.shape)
        sl_lo, sl_hi = [slice(None)] * 3, [slice(None)] * 3
        sl_lo[ax], sl_hi[ax] = slice(None, -1), slice(1, None)
        a2[tuple(sl_lo)] = a[tuple(sl_hi)]
        f2[tuple(sl_lo)] = f[tuple(sl_hi)]
        s = a + a2
        out.append(np.where(s > 0, (a * f + a2 * f2) / np.where(s > 0, s, 1.0), 0.0))
    return out


def wall_shear_stress(u, v, w, st, nu):
    """The resolved nu |u_t(image)| / probe at every stencil."""
    uc, vc, wc = (a.ravel() for a in center_velocity(u, v, w, st.geom))
    tau = np.zeros(len(st))
    for s in range(len(st)):
        if not st.valid[s]:
            continue
        ui = image_value(uc, st.donors[s], st.weights[s])
        vi = image_value(vc, st.donors[s], st.weights[s])
        wi = image_value(wc, st.donors[s], st.weights[s])
        n = st.normal[s]
        un = ui * n[0] + vi * n[1] + wi * n[2]
        t2 = ui * ui + vi * vi + wi * wi - un * un
        tau[s] = nu * math.sqrt(max(t2, 0.0)) / st.probe[s]
    return tau


# ----------------------------------------------------------------------------- laws
def exp_tail(x, m):
    if abs(x) < 0.5:
        term = x ** m / math.factorial(m)
        s = term
        n = m
        while abs(term) > EPS * abs(s) / 4:
            n += 1
            term *= x / n
            s += term
        return s
    s = math.expm1(x) - x - x * x / 2
    return s if m == 3 else s - x ** 3 / 6


def spalding_yplus(kappa, B, up):
    return up + math.exp(-kappa * B) * exp_tail(kappa * up, 4)


def spalding_dyplus(kappa, B, up):
    return 1 + kappa * math.exp(-kappa * B) * exp_tail(kappa * up, 3)


def increasing_root(fg, lo, hi, x, maxiter=200):
    for _ in range(maxiter):
        f, g = fg(x)
        if not math.isfinite(f) or f > 0:
            hi = x
        elif f < 0:
            lo = x
        else:
            return x
        xn = x - f / g if (math.isfinite(f) and g > 0) else (lo + hi) / 2
        if not (lo < xn < hi):
            xn = (lo + hi) / 2
        if abs(xn - x) <= 2 * EPS * abs(xn):
            return xn
        x = xn
    return x


def psi_m(zeta):
    if zeta < 0:
        x = (1 - 16.0 * zeta) ** 0.25
        return 2 * math.log((1 + x) / 2) + math.log((1 + x * x) / 2) - 2 * math.atan(x) + math.pi / 2
    a, b, c, d = 1.0, 2 / 3, 5.0, 0.35
    return -(a * zeta + b * (zeta - c / d) * math.exp(-d * zeta) + b * c / d)


def friction_velocity(law, U, h, nu=None):
    name = type(law).__name__
    if name == "SpaldingLaw":
        a = abs(U)
        if not a > 0:
            return 0.0
        Re = a * h / nu
        hi = math.sqrt(Re)
        x0 = hi
        if Re > 1:
            x0 = 10.0
            for _ in range(3):
                x0 = max(math.log(Re / x0) / law.kappa + law.B, 1.0)
            x0 = min(x0, hi)

        def fg(up):
            y = spalding_yplus(law.kappa, law.B, up)
            return up * y - Re, y + up * spalding_dyplus(law.kappa, law.B, up)
        return a / increasing_root(fg, 0.0, hi, x0)
    if name == "RoughLogLaw":
        return law.kappa * abs(U) / math.log(h / law.z0)
    if name == "MOSTWallLaw":
        Ue = max(math.sqrt(U * U), law.U_min)
        zeta = h / law.L
        phim = math.log(h / law.z0m) - psi_m(zeta) + psi_m(zeta * law.z0m / h)
        return law.kappa * Ue / phim
    raise ValueError(name)


def wall_stress_and_slip(u, v, w, st, law, nu=None, nu_eff=None):
    """wall_shear_stress(..., law) and wall_slip_velocity(..., law; nu, nu_eff)."""
    uc, vc, wc = (a.ravel() for a in center_velocity(u, v, w, st.geom))
    n = len(st)
    tau = np.zeros(n)
    slip = np.zeros((n, 3))
    for s in range(n):
        if not st.valid[s]:
            continue
        ui = image_value(uc, st.donors[s], st.weights[s])
        vi = image_value(vc, st.donors[s], st.weights[s])
        wi = image_value(wc, st.donors[s], st.weights[s])
        nv = st.normal[s]
        un = ui * nv[0] + vi * nv[1] + wi * nv[2]
        t = (ui - un * nv[0], vi - un * nv[1], wi - un * nv[2])
        ut = math.sqrt(t[0] ** 2 + t[1] ** 2 + t[2] ** 2)
        ts = friction_velocity(law, ut, st.probe[s], nu) ** 2
        tau[s] = ts
        if ut != 0:
            r = (ut - ts * st.probe[s] / nu_eff) / ut
            slip[s] = (r * t[0], r * t[1], r * t[2])
    return tau, slip
