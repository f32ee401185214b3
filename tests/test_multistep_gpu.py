"""n steps as one graph launch: `step_rk3(dt, n)` runs the step pairs as a
conditional WHILE node over a captured two-step body (the state sets swap
back after each pair) and any odd step on its own.  It must equal n calls of
one step bit for bit: the same kernels in the same order, on the column,
FFT and cut-cell MG-PCG projections (the last with its CG loops as
conditional nodes nested in the loop body)."""
import numpy as np
import pytest

from aeolus_b200 import CoreSpec, regular_grid, stretched_grid, tanh_beta_for_first_cell, tanh_faces
from aeolus_b200.cutcell import box_solid_mask, face_coefficients, random_boxes, staircase_geometry
from aeolus_b200.inputs import cbl_initial, cbl_theta_profile, taylor_green
from aeolus_b200.reference_state import anelastic_profiles, exponential_density

pytestmark = pytest.mark.gpu

FIELDS = ("u", "v", "w", "theta")


def pair(spec, state, setup=None):
    from aeolus_b200.simulation import Simulation
    sims = [Simulation(spec), Simulation(spec)]
    for s in sims:
        if setup:
            setup(s)
        s.set_state(*state)
    return sims


def same(a, b):
    for n in FIELDS:
        assert np.array_equal(a.get_field(n), b.get_field(n)), n


@pytest.mark.parametrize("n", [6, 7])
def test_multistep_equals_single_steps_column(n):
    nz = 32
    g = stretched_grid((32, 32, nz), (640.0, 640.0, 2000.0), tanh_faces(nz, 2000.0, tanh_beta_for_first_cell(nz, 2000.0, 32.0)))
    prof = anelastic_profiles(g, exponential_density(g), cbl_theta_profile(g.znodes("c")))
    sp = CoreSpec(grid=g, core="anelastic", c_s=0.17, flux_bot=0.1, wc=prof["wc"], wf=prof["wf"], thf=prof["thf"])
    u, v, w, th, _ = cbl_initial(g, seed=1, noise=0.1)
    a, b = pair(sp, (u, v, w, th))
    a.step_rk3(1.0, n)
    for _ in range(n):
        b.step_rk3(1.0, 1)
    same(a, b)


def test_multistep_equals_single_steps_fft_fp32():
    g = regular_grid((32, 32, 32), (2 * np.pi,) * 3)
    sp = CoreSpec(grid=g, advection="weno_z5", nu=1e-3, precision="fp32_mixed")
    a, b = pair(sp, taylor_green(g, seed=1, amp=1e-3))
    a.step_rk3(0.01, 5)
    for _ in range(5):
        b.step_rk3(0.01, 1)
    same(a, b)


def test_multistep_equals_single_steps_pcg():
    g = regular_grid((32, 32, 16), (64.0, 64.0, 32.0), halo=(3, 3, 3), bc_z="wall")
    geom = staircase_geometry(g, box_solid_mask(g, random_boxes(g, 4, seed=2, footprint=(8.0, 16.0),
                                                                   height=(6.0, 20.0))))
    ap = face_coefficients(geom, power=1)
    nx, ny, nz = g.size
    th = np.full(g.storage_shape, 300.0)
    th[g.interior] += 0.1 * (2 * np.random.default_rng(1).random((nz, ny, nx)) - 1)
    z = g.zeros()
    sp = CoreSpec(grid=g, c_s=0.17, theta0=300.0, flux_bot=0.15, solver="pcg", precision="fp32_mixed")
    a, b = pair(sp, (z, z, z, th), setup=lambda s: s.set_pcg(ap, tol=1e-8, maxit=300))
    a.step_rk3(1.0, 4)
    for _ in range(4):
        b.step_rk3(1.0, 1)
    same(a, b)
    assert a.pcg_stats()["status"] == "converged"
