"""The oracle's positivity-preserving advection (advect_positive!,
src/AdvectionSchemes.jl:1100-1160) on the CPU.

Restates the reference's guarantees and checks:
  * a forward-Euler update with the same dt keeps a non-negative field
    non-negative when sum_d |u_d| dt/dx_d <= 1 (the docstring's contract,
    and the positivity test of test/advection.jl), where the unlimited
    WENO-Z5 update undershoots;
  * the flux form conserves the field's sum (periodic domain, walls);
  * where nothing can go negative the limiter is inactive and the tendency
    is the reconstructed flux divergence of the step's own WENO advection.
"""
import numpy as np
import pytest

from oracle.oracle import OracleSimulation
from positive_cases import case, grid, spec


@pytest.mark.parametrize("scheme", ["weno_z5", "weno_js5"])
@pytest.mark.parametrize("bc_z", ["periodic", "wall"])
def test_positive_and_conservative(scheme, bc_z):
    g = grid(bc_z=bc_z)
    o = OracleSimulation(spec(g))
    u, v, w, phi, dt = case(g, 3)
    tend = o.advect_positive(u, v, w, phi, dt, scheme=scheme, accumulate=False)[g.interior]
    new = phi[g.interior] + dt * tend
    assert new.min() >= -1e-14 * phi.max()
    assert abs(tend.sum()) <= 1e-12 * np.abs(tend).sum()


def test_unlimited_weno_undershoots_where_the_limiter_holds():
    g = grid()
    o = OracleSimulation(spec(g))
    u, v, w, phi, dt = case(g, 4)
    sp = spec(g)
    sp.nu = 0.0
    ref = OracleSimulation(sp)
    ref.set_state(u, v, w, phi)
    plain = -ref.tendencies()[3][g.interior]   # the step's WENO-Z5 flux divergence, -(-div(u phi))
    assert (phi[g.interior] - dt * plain).min() < -1e-3
    lim = o.advect_positive(u, v, w, phi, dt, accumulate=False)[g.interior]
    assert (phi[g.interior] + dt * lim).min() >= -1e-14


def test_limiter_inactive_on_a_smooth_positive_field():
    g = grid()
    o = OracleSimulation(spec(g))
    u, v, w, phi, dt = case(g, 5, cfl=0.2, sharp=False)
    sp = spec(g)
    sp.nu = 0.0
    ref = OracleSimulation(sp)
    ref.set_state(u, v, w, phi)
    tt = ref.tendencies()[3][g.interior]
    lim = o.advect_positive(u, v, w, phi, dt, accumulate=False)[g.interior]
    assert np.abs(lim - tt).max() <= 1e-12 * np.abs(tt).max()


def test_accumulate_adds_to_the_given_tendency():
    g = grid()
    o = OracleSimulation(spec(g))
    u, v, w, phi, dt = case(g, 6)
    base = np.random.default_rng(7).standard_normal(g.storage_shape)
    a = o.advect_positive(u, v, w, phi, dt, tend=base, accumulate=True)
    b = o.advect_positive(u, v, w, phi, dt, accumulate=False)
    assert np.allclose(a[g.interior], base[g.interior] + b[g.interior], rtol=0, atol=1e-13)
