"""The Vreman (2004) SGS closure (VremanClosure / compute_vreman_nut!,
src/operators/sgs_amd_vreman.jl:93-100, :280-298, :370-380): nu_t =
2.5 c_s^2 sqrt(B_beta / alpha:alpha) from the velocity-gradient stencil of
the Smagorinsky closure, kappa_t = nu_t / Pr_t.

Oracle (CPU): nu_t equals a numpy statement of _vreman_point on a random
field; it is exactly zero in a pure shear flow u(z) (B_beta vanishes when
the velocity varies in one direction, the closure's design property) where
Smagorinsky's is not.  GPU (`-m gpu`): steps with the Vreman closure match
the oracle to 1e-11 (FP64) and FP32-mixed to 1e-5.
"""
import numpy as np
import pytest

from aeolus_b200 import CoreSpec, regular_grid
from oracle.oracle import OracleSimulation

FIELDS = ("u", "v", "w", "theta")


def grid():
    return regular_grid((16, 16, 16), (1.0, 1.0, 0.5), halo=(3, 3, 3), bc_z="wall")


def spec(g, sgs="vreman", advection="centred", precision="fp64"):
    return CoreSpec(grid=g, c_s=0.17, sgs=sgs, theta0=300.0, advection=advection, precision=precision)


def state(g, seed=4):
    rng = np.random.default_rng(seed)
    nx, ny, nz = g.size
    th = np.full(g.storage_shape, 300.0)
    th[g.interior] += 0.1 * rng.standard_normal((nz, ny, nx))
    u, v, w = g.zeros(), g.zeros(), g.zeros()
    u[g.interior] = rng.standard_normal((nz, ny, nx))
    v[g.interior] = rng.standard_normal((nz, ny, nx))
    w[g.interior] = rng.standard_normal((nz, ny, nx))
    w[g.halo[2]] = 0.0
    return u, v, w, th


def vreman_numpy(g, u, v, w, c_s):
    """_velocity_gradient_at and _vreman_point on the interior (storage arrays with filled halos)."""
    hx, hy, hz = g.halo
    nx, ny, nz = g.size
    K, J, I = slice(hz, hz + nz), slice(hy, hy + ny), slice(hx, hx + nx)

    def sh(a, di, dj, dk):
        return a[hz + dk:hz + dk + nz, hy + dj:hy + dj + ny, hx + di:hx + di + nx]
    idx, idy, idz = 1 / g.dx, 1 / g.dy, 1 / g.dz
    du_dx = (sh(u, 1, 0, 0) - sh(u, 0, 0, 0)) * idx
    dv_dy = (sh(v, 0, 1, 0) - sh(v, 0, 0, 0)) * idy
    dw_dz = (sh(w, 0, 0, 1) - sh(w, 0, 0, 0)) * idz
    du_dy = ((sh(u, 0, 1, 0) + sh(u, 1, 1, 0)) - (sh(u, 0, -1, 0) + sh(u, 1, -1, 0))) * (0.25 * idy)
    dv_dx = ((sh(v, 1, 0, 0) + sh(v, 1, 1, 0)) - (sh(v, -1, 0, 0) + sh(v, -1, 1, 0))) * (0.25 * idx)
    du_dz = ((sh(u, 0, 0, 1) + sh(u, 1, 0, 1)) - (sh(u, 0, 0, -1) + sh(u, 1, 0, -1))) * (0.25 * idz)
    dw_dx = ((sh(w, 1, 0, 0) + sh(w, 1, 0, 1)) - (sh(w, -1, 0, 0) + sh(w, -1, 0, 1))) * (0.25 * idx)
    dv_dz = ((sh(v, 0, 0, 1) + sh(v, 0, 1, 1)) - (sh(v, 0, 0, -1) + sh(v, 0, 1, -1))) * (0.25 * idz)
    dw_dy = ((sh(w, 0, 1, 0) + sh(w, 0, 1, 1)) - (sh(w, 0, -1, 0) + sh(w, 0, -1, 1))) * (0.25 * idy)
    a1 = np.stack([du_dx, dv_dx, dw_dx])
    a2 = np.stack([du_dy, dv_dy, dw_dy])
    a3 = np.stack([du_dz, dv_dz, dw_dz])

    def cross2(a, b):
        return (np.cross(a, b, axis=0) ** 2).sum(axis=0)
    Bb = (g.dx ** 2 * g.dy ** 2 * cross2(a1, a2) + g.dx ** 2 * g.dz ** 2 * cross2(a1, a3)
          + g.dy ** 2 * g.dz ** 2 * cross2(a2, a3))
    aa = (a1 ** 2).sum(axis=0) + (a2 ** 2).sum(axis=0) + (a3 ** 2).sum(axis=0)
    return np.where(aa > 0, 2.5 * c_s ** 2 * np.sqrt(Bb / np.where(aa > 0, aa, 1.0)), 0.0)


def test_oracle_nut_is_the_vreman_point():
    g = grid()
    o = OracleSimulation(spec(g))
    o.set_state(*state(g))
    o.tendencies()
    nut = o.get_field("nut")[g.interior]
    u, v, w = (o.get_field(n) for n in ("u", "v", "w"))
    ref = vreman_numpy(g, u, v, w, 0.17)
    assert np.abs(nut - ref).max() <= 1e-13 * np.abs(ref).max()


def test_vreman_vanishes_in_pure_shear():
    g = grid()
    z = g.znodes("c")
    u = g.zeros()
    u[g.interior] = np.sin(3 * z)[:, None, None]
    zero = g.zeros()
    th = np.full(g.storage_shape, 300.0)
    for sgs, expect_zero in (("vreman", True), ("smagorinsky", False)):
        o = OracleSimulation(spec(g, sgs))
        o.set_state(u, zero, zero, th)
        o.tendencies()
        nut = o.get_field("nut")[g.interior]
        assert (np.abs(nut).max() == 0.0) == expect_zero, sgs


def test_vreman_needs_a_uniform_grid():
    from aeolus_b200 import stretched_grid, tanh_faces
    g = stretched_grid((16, 16, 16), (1.0, 1.0, 0.5), tanh_faces(16, 0.5, 1.5), halo=(3, 3, 3))
    with pytest.raises(ValueError):
        CoreSpec(grid=g, c_s=0.17, sgs="vreman")


@pytest.mark.gpu
@pytest.mark.parametrize("advection", ["centred", "weno_js5"])
def test_gpu_vreman_steps_match_the_oracle(advection):
    from aeolus_b200.simulation import Simulation
    g = grid()
    st = state(g)
    sims = [OracleSimulation(spec(g, advection=advection)), Simulation(spec(g, advection=advection)),
            Simulation(spec(g, advection=advection, precision="fp32_mixed"))]
    out = []
    for s in sims:
        s.set_state(*st)
        s.project()
        s.step_rk3(2e-3, 3)
        out.append({n: s.get_field(n)[g.interior] for n in FIELDS})
    ora, g64, g32 = out
    e64 = {n: np.linalg.norm(g64[n] - ora[n]) / np.linalg.norm(ora[n]) for n in FIELDS}
    assert all(e <= 1e-11 for e in e64.values()), e64
    e32 = {n: np.linalg.norm(g32[n] - g64[n]) / np.linalg.norm(g64[n]) for n in FIELDS}
    assert all(e <= 1e-5 for e in e32.values()), e32
    nut = sims[1].get_field("nut")[g.interior]
    ref = vreman_numpy(g, *(sims[1].get_field(n) for n in ("u", "v", "w")), 0.17)
    assert np.abs(nut - ref).max() <= 1e-12 * np.abs(ref).max()
