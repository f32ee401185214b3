"""The density-weighted cut-cell projection on the sound-proof core and on a
stretched column (solver = "pcg" with core = "anelastic" or a tanh column).

The MG-preconditioned CG solves D(W a^2 G phi) = D(W a u*) with the weights of
DensityWeightedPoissonSolver (src/Anelastic.jl:734-793: W_c on the x and y
faces, W_f on the z faces) and the aperture form of the cut-cell operators
(src/CutCell.jl:602-700), every equation taken times dz_c / h_z so that the
stretched operator is the symmetric face-coefficient form the multigrid
hierarchy coarsens.  With every face open this is the direct weighted
column solve of the same core (DirectWeightedPoissonSolver,
src/Anelastic.jl:987-1021, composed with the stretched metrics), so the two
projected steps agree to the CG tolerance; with buildings the projected
velocity has zero density- and aperture-weighted divergence and no flow
through a blocked face.  CPU tests use the oracle; `-m gpu` tests compare the
CUDA step with it."""
import numpy as np
import pytest

from aeolus_b200 import CoreSpec, stretched_grid, tanh_beta_for_first_cell, tanh_faces
from aeolus_b200.cutcell import box_solid_mask, face_coefficients, random_boxes, staircase_geometry
from aeolus_b200.reference_state import anelastic_profiles, exponential_density
from oracle.oracle import OracleSimulation

N = (32, 32, 24)
LZ = 96.0
FIELDS = ("u", "v", "w", "theta")


def grid():
    nz = N[2]
    return stretched_grid(N, (64.0, 64.0, LZ), tanh_faces(nz, LZ, tanh_beta_for_first_cell(nz, LZ, 2.0)))


def theta_profile(z):
    return 300.0 + 0.01 * z            # a weakly stable column


def spec(g, core, solver, precision="fp64"):
    if core == "anelastic":
        prof = anelastic_profiles(g, exponential_density(g), theta_profile(g.znodes("c")))
        return CoreSpec(grid=g, core="anelastic", nu=1e-3, c_s=0.17, flux_bot=0.1, solver=solver,
                        precision=precision, wc=prof["wc"], wf=prof["wf"], thf=prof["thf"])
    # no buoyancy on the Boussinesq column: against a constant theta0 the
    # stratified theta is a hydrostatic source far larger than the flow's, and
    # a relative CG tolerance of it says little about the small projected w
    return CoreSpec(grid=g, nu=1e-3, c_s=0.17, theta0=0.0, flux_bot=0.1, solver=solver, precision=precision)


def staircase(g):
    geom = staircase_geometry(g, box_solid_mask(g, random_boxes(g, 4, seed=2, footprint=(8.0, 16.0),
                                                                   height=(6.0, 20.0))))
    return geom, face_coefficients(geom, power=1)


def state(g, seed, fluid=None):
    rng = np.random.default_rng(seed)
    nx, ny, nz = g.size
    th = np.broadcast_to(theta_profile(g.znodes("c"))[:, None, None], (nz, ny, nx)) + \
        0.1 * rng.standard_normal((nz, ny, nx))
    u, v, t = g.zeros(), g.zeros(), g.zeros()
    u[g.interior] = 1.0 + 0.1 * rng.standard_normal((nz, ny, nx))
    v[g.interior] = 0.1 * rng.standard_normal((nz, ny, nx))
    t[g.interior] = th
    if fluid is not None:
        u[g.interior] *= fluid
        v[g.interior] *= fluid
    return u, v, g.zeros(), t


def rel_l2(a, b, g):
    a, b = a[g.interior], b[g.interior]
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("core", ["anelastic", "boussinesq"])
def test_open_weighted_pcg_step_equals_the_column_step(core):
    g = grid()
    col, pcg = OracleSimulation(spec(g, core, "column")), OracleSimulation(spec(g, core, "pcg"))
    pcg.set_pcg(None, tol=1e-13, maxit=500)
    st = state(g, 3)
    for s in (col, pcg):
        s.set_state(*st)
        s.project()
        s.step_rk3(0.5, 3)
    errs = {n: rel_l2(pcg.get_field(n), col.get_field(n), g) for n in FIELDS}
    assert all(e <= 1e-10 for e in errs.values()), errs
    assert pcg.pcg_stats()["status"] == "converged"
    assert pcg.max_divergence() < 1e-10


def test_weighted_projection_around_buildings():
    g = grid()
    geom, ap = staircase(g)
    fluid = (~geom.is_solid[g.interior]).astype(float)
    s = OracleSimulation(spec(g, "anelastic", "pcg"))
    s.set_pcg(ap, tol=1e-12, maxit=500)
    s.set_state(*state(g, 5, fluid))
    s.project()
    s.step_rk3(0.5, 2)
    assert s.pcg_stats()["status"] == "converged"
    assert s.max_divergence() < 1e-9
    hx, hy, hz = g.halo
    nx, ny, nz = g.size
    u = s.get_field("u")[hz:hz + nz, hy:hy + ny, hx:hx + nx]
    assert np.abs(u[ap[0][:, :, :nx] == 0]).max() == 0.0      # no flow through a blocked face


# ------------------------------------------------------------------ GPU ---
@pytest.mark.gpu
@pytest.mark.parametrize("core", ["anelastic", "boussinesq"])
def test_gpu_weighted_pcg_step_with_buildings_matches_the_oracle(core):
    from aeolus_b200.simulation import Simulation
    g = grid()
    geom, ap = staircase(g)
    fluid = (~geom.is_solid[g.interior]).astype(float)
    gpu, ora = Simulation(spec(g, core, "pcg")), OracleSimulation(spec(g, core, "pcg"))
    st = state(g, 11, fluid)
    for s in (gpu, ora):
        s.set_pcg(ap, tol=1e-12, maxit=500)
        s.set_state(*st)
        s.project()
        s.step_rk3(0.5, 3)
    errs = {n: rel_l2(gpu.get_field(n), ora.get_field(n), g) for n in FIELDS}
    assert all(e <= 1e-10 for e in errs.values()), errs
    a, b = gpu.pcg_stats(), ora.pcg_stats()
    assert a["status"] == b["status"] == "converged"
    assert abs(a["iterations"] - b["iterations"]) <= 1, (a, b)
    assert gpu.max_divergence() < 1e-9


@pytest.mark.gpu
def test_gpu_open_weighted_pcg_step_equals_the_column_step():
    from aeolus_b200.simulation import Simulation
    g = grid()
    col, pcg = Simulation(spec(g, "anelastic", "column")), Simulation(spec(g, "anelastic", "pcg"))
    pcg.set_pcg(None, tol=1e-13, maxit=500)
    st = state(g, 3)
    for s in (col, pcg):
        s.set_state(*st)
        s.project()
        s.step_rk3(0.5, 3)
    errs = {n: rel_l2(pcg.get_field(n), col.get_field(n), g) for n in FIELDS}
    assert all(e <= 1e-9 for e in errs.values()), errs


@pytest.mark.gpu
def test_gpu_fp32_mixed_weighted_pcg_step_close_to_fp64():
    from aeolus_b200.simulation import Simulation
    g = grid()
    geom, ap = staircase(g)
    fluid = (~geom.is_solid[g.interior]).astype(float)
    sims = [Simulation(spec(g, "anelastic", "pcg", p)) for p in ("fp64", "fp32_mixed")]
    st = state(g, 7, fluid)
    for s in sims:
        s.set_pcg(ap, tol=1e-10, maxit=500)
        s.set_state(*st)
        s.project()
        s.step_rk3(0.5, 5)
    errs = {n: rel_l2(sims[1].get_field(n), sims[0].get_field(n), g) for n in ("u", "v", "w")}
    th0 = st[3][g.interior]
    a, b = sims[1].get_field("theta")[g.interior] - th0, sims[0].get_field("theta")[g.interior] - th0
    errs["theta_departure"] = np.linalg.norm(a - b) / np.linalg.norm(b)
    assert all(e <= 1e-5 for e in errs.values()), errs
