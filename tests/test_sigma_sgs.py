"""The sigma-model SGS closure (SigmaModel / compute_sigma_nut!,
src/operators/sigma_closure.jl:130-222): nu_t = (C_sigma Delta)^2 D_sigma,
D_sigma = s3 (s1 - s2)(s2 - s3) / s1^2 of the singular values of the
velocity-gradient tensor (the Smagorinsky stencil), kappa_t = nu_t / Pr_t.

Oracle (CPU): nu_t equals (C Delta)^2 D_sigma from numpy's SVD of the same
gradients on a random field; it vanishes exactly for a gradient of rank <= 2
(a two-dimensional flow) -- the closure's design property, which the closed
form keeps by taking s3 from the determinant.  GPU (`-m gpu`): steps with the
sigma closure match the oracle (1e-10 FP64, 1e-5 FP32-mixed).
"""
import numpy as np
import pytest

from aeolus_b200 import CoreSpec, regular_grid
from oracle.oracle import OracleSimulation
from test_vreman import state

FIELDS = ("u", "v", "w", "theta")
C_SIGMA = 1.35


def grid():
    return regular_grid((16, 16, 16), (1.0, 1.0, 0.5), halo=(3, 3, 3), bc_z="wall")


def spec(g, advection="centred", precision="fp64"):
    return CoreSpec(grid=g, c_s=C_SIGMA, sgs="sigma", theta0=300.0, advection=advection, precision=precision)


def gradients(g, u, v, w):
    hx, hy, hz = g.halo
    nx, ny, nz = g.size

    def sh(a, di, dj, dk):
        return a[hz + dk:hz + dk + nz, hy + dj:hy + dj + ny, hx + di:hx + di + nx]
    idx, idy, idz = 1 / g.dx, 1 / g.dy, 1 / g.dz
    G = np.empty((nz, ny, nx, 3, 3))
    G[..., 0, 0] = (sh(u, 1, 0, 0) - sh(u, 0, 0, 0)) * idx
    G[..., 1, 1] = (sh(v, 0, 1, 0) - sh(v, 0, 0, 0)) * idy
    G[..., 2, 2] = (sh(w, 0, 0, 1) - sh(w, 0, 0, 0)) * idz
    G[..., 0, 1] = ((sh(u, 0, 1, 0) + sh(u, 1, 1, 0)) - (sh(u, 0, -1, 0) + sh(u, 1, -1, 0))) * (0.25 * idy)
    G[..., 1, 0] = ((sh(v, 1, 0, 0) + sh(v, 1, 1, 0)) - (sh(v, -1, 0, 0) + sh(v, -1, 1, 0))) * (0.25 * idx)
    G[..., 0, 2] = ((sh(u, 0, 0, 1) + sh(u, 1, 0, 1)) - (sh(u, 0, 0, -1) + sh(u, 1, 0, -1))) * (0.25 * idz)
    G[..., 2, 0] = ((sh(w, 1, 0, 0) + sh(w, 1, 0, 1)) - (sh(w, -1, 0, 0) + sh(w, -1, 0, 1))) * (0.25 * idx)
    G[..., 1, 2] = ((sh(v, 0, 0, 1) + sh(v, 0, 1, 1)) - (sh(v, 0, 0, -1) + sh(v, 0, 1, -1))) * (0.25 * idz)
    G[..., 2, 1] = ((sh(w, 0, 1, 0) + sh(w, 0, 1, 1)) - (sh(w, 0, -1, 0) + sh(w, 0, -1, 1))) * (0.25 * idy)
    return G


def sigma_numpy(g, u, v, w):
    s = np.linalg.svd(gradients(g, u, v, w), compute_uv=False)
    s1, s2, s3 = s[..., 0], s[..., 1], s[..., 2]
    D = np.where(s1 > 0, s3 * (s1 - s2) * (s2 - s3) / np.where(s1 > 0, s1 * s1, 1.0), 0.0)
    delta = (g.dx * g.dy * g.dz) ** (1 / 3)
    return (C_SIGMA * delta) ** 2 * np.maximum(D, 0.0)


def test_oracle_nut_is_the_sigma_operator():
    g = grid()
    o = OracleSimulation(spec(g))
    o.set_state(*state(g))
    o.tendencies()
    nut = o.get_field("nut")[g.interior]
    u, v, w = (o.get_field(n) for n in ("u", "v", "w"))
    ref = sigma_numpy(g, u, v, w)
    assert np.abs(nut - ref).max() <= 1e-9 * np.abs(ref).max()
    assert (nut > 0).mean() > 0.9


def test_sigma_vanishes_for_a_two_dimensional_flow():
    g = grid()
    rng = np.random.default_rng(5)
    nx, ny, nz = g.size
    u, v, w = g.zeros(), g.zeros(), g.zeros()
    # u(x, y), v(x, y), w = 0: the z row and column of the gradient vanish (rank <= 2)
    u2 = rng.standard_normal((ny, nx))
    v2 = rng.standard_normal((ny, nx))
    u[g.interior] = u2[None]
    v[g.interior] = v2[None]
    th = np.full(g.storage_shape, 300.0)
    o = OracleSimulation(spec(g))
    o.set_state(u, v, w, th)
    o.tendencies()
    assert np.abs(o.get_field("nut")[g.interior]).max() == 0.0


@pytest.mark.gpu
@pytest.mark.parametrize("advection", ["centred", "weno_js5"])
def test_gpu_sigma_steps_match_the_oracle(advection):
    from aeolus_b200.simulation import Simulation
    g = grid()
    st = state(g)
    sims = [OracleSimulation(spec(g, advection)), Simulation(spec(g, advection)),
            Simulation(spec(g, advection, "fp32_mixed"))]
    out = []
    for s in sims:
        s.set_state(*st)
        s.project()
        s.step_rk3(2e-3, 3)
        out.append({n: s.get_field(n)[g.interior] for n in FIELDS})
    ora, g64, g32 = out
    e64 = {n: np.linalg.norm(g64[n] - ora[n]) / np.linalg.norm(ora[n]) for n in FIELDS}
    assert all(e <= 1e-10 for e in e64.values()), e64
    e32 = {n: np.linalg.norm(g32[n] - g64[n]) / np.linalg.norm(g64[n]) for n in FIELDS}
    assert all(e <= 1e-5 for e in e32.values()), e32
    nut = sims[1].get_field("nut")[g.interior]
    ref = sigma_numpy(g, *(sims[1].get_field(n) for n in ("u", "v", "w")))
    assert np.abs(nut - ref).max() <= 1e-9 * np.abs(ref).max()
