"""The oracle pinned against the reference's own known answers and analytic
tests (CPU only).

Julia is not available, so the reference cannot be executed; its tests are
restated here against the oracle:
  * Philox4x32-10 Random123 KATs          test/backends.jl:269-273
  * manufactured Poisson solutions         test/runtests.jl:168-260
  * column solver = transform solve,
    incompatible source -> uniform -mean   test/pressure_column.jl:30-60
  * round-off divergence after a step      test/ka_step.jl:117-120
  * RK3 third order in time (TGV)          test/ka_step.jl:121-136
  * TGV decay at the 7-point rate          test/ka_step.jl:137-147
  * WENO design order                      test/advection.jl:52-100
  * anelastic: hydrostatic rest state,
    constraint at round-off                test/anelastic.jl:39-180
"""
import json
import os

import numpy as np
import pytest

from aeolus_b200 import CoreSpec, regular_grid, stretched_grid, tanh_faces
from aeolus_b200.inputs import philox4x32 as np_philox
from aeolus_b200.inputs import philox_uniform, taylor_green
from aeolus_b200.reference_state import anelastic_profiles, exponential_density
from oracle.oracle import OracleSimulation, philox4x32, uniform_fill

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def load_golden(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


# ---------------------------------------------------------------- Philox ----
def test_philox_known_answers():
    kat = load_golden("philox4x32_10_kat.json")
    assert len(kat["vectors"]) == 3
    for v in kat["vectors"]:
        ctr = [int(x, 16) for x in v["ctr"]]
        key = [int(x, 16) for x in v["key"]]
        out = tuple(int(x, 16) for x in v["out"])
        assert philox4x32(ctr, key) == out
        assert tuple(int(np.asarray(c)) for c in np_philox(ctr, key)) == out


def test_philox_uniform_stream_matches_numpy():
    a = uniform_fill(2026, 3, 5000, 1.0)
    b = 2 * philox_uniform(2026, 3, 5000) - 1
    assert np.array_equal(a, b)
    # first draws of neighbouring streams are uniform (4 sigma), test/backends.jl:281-282
    xs = philox_uniform(2026, 0, 20000)
    assert abs(xs.mean() - 0.5) < 4 * np.sqrt(1 / 12 / len(xs))


# ---------------------------------------------------------------- Poisson ---
def _rand(shape, seed):
    return np.random.default_rng(seed).standard_normal(shape)


def test_fft_poisson_manufactured():
    g = regular_grid((16, 12, 8), (1.0, 2.0, 3.0))
    o = OracleSimulation(CoreSpec(grid=g))
    phi = _rand((8, 12, 16), 1)
    phi -= phi.mean()
    sol = o.pressure_solve(o.apply_poisson_operator(phi))
    assert np.abs(sol - phi).max() < 1e-12 * np.abs(phi).max()
    assert abs(sol.mean()) < 1e-13


@pytest.mark.parametrize("stretched", [False, True])
def test_column_poisson_manufactured_and_gauge(stretched):
    nz = 12
    if stretched:
        g = stretched_grid((16, 8, nz), (400.0, 200.0, 300.0), tanh_faces(nz, 300.0, 1.8))
    else:
        g = regular_grid((16, 8, nz), (400.0, 200.0, 300.0), bc_z="wall")
    o = OracleSimulation(CoreSpec(grid=g))
    phi = _rand((nz, 8, 16), 2)
    sol = o.pressure_solve(o.apply_poisson_operator(phi))
    d = sol - phi
    assert np.abs(d - d.mean()).max() < 1e-11 * np.abs(phi).max()
    dzc = g.cell_thickness()
    # zero volume-weighted mean gauge (src/PressureSolvers.jl:780-805)
    assert abs((sol.sum(axis=(1, 2)) * dzc).sum()) < 1e-10 * np.abs(sol).max() * dzc.sum()


def test_column_incompatible_source_residual_is_uniform_minus_mean():
    g = regular_grid((16, 8, 12), (480.0, 400.0, 160.0), bc_z="wall")
    o = OracleSimulation(CoreSpec(grid=g))
    raw = _rand((12, 8, 16), 5) + 0.3
    p = o.pressure_solve(raw)
    r = o.apply_poisson_operator(p) - raw
    assert np.abs(r + raw.mean()).max() < 1e-10


def test_column_equals_fft_transform_solve_when_z_is_periodic_equivalent():
    # The column (Thomas) path and the all-transform path solve the same
    # discrete problem: compare the column solver against the dense solve of
    # its own operator on a small grid.
    g = regular_grid((8, 4, 6), (8.0, 4.0, 6.0), bc_z="wall")
    o = OracleSimulation(CoreSpec(grid=g))
    n = 8 * 4 * 6
    Amat = np.empty((n, n))
    for c in range(n):
        e = np.zeros(n)
        e[c] = 1.0
        Amat[:, c] = o.apply_poisson_operator(e.reshape(6, 4, 8)).ravel()
    src = _rand((6, 4, 8), 9)
    src -= src.mean()
    sol = o.pressure_solve(src).ravel()
    ref = np.linalg.lstsq(Amat, src.ravel(), rcond=None)[0]
    ref -= ref.mean()
    assert np.abs((sol - sol.mean()) - ref).max() < 1e-11 * np.abs(ref).max()


def test_anelastic_weighted_column_solver():
    nz = 16
    g = stretched_grid((16, 8, nz), (320.0, 160.0, 400.0), tanh_faces(nz, 400.0, 1.2))
    rho = exponential_density(g)
    prof = anelastic_profiles(g, rho, np.full(nz, 300.0))
    o = OracleSimulation(CoreSpec(grid=g, core="anelastic", wc=prof["wc"], wf=prof["wf"], thf=prof["thf"]))
    phi = _rand((nz, 8, 16), 3)
    sol = o.pressure_solve(o.apply_poisson_operator(phi))
    d = sol - phi
    assert np.abs(d - d.mean()).max() < 1e-10 * np.abs(phi).max()


# ---------------------------------------------------------------- steps -----
def test_divergence_round_off_after_step_from_random_start():
    n = 16
    g = regular_grid((n, n, n), (2 * np.pi,) * 3)
    o = OracleSimulation(CoreSpec(grid=g, nu=1e-2))
    for k, name in enumerate(("u", "v", "w")):
        a = g.zeros()
        a[g.interior] = _rand((n, n, n), 404 + k)
        o.set_field(name, a)
    o.step(0.05)
    assert o.max_divergence() < 1e-12


def _tg(g, nu, dt, U=1.0, T=1.0, scheme="centred"):
    o = OracleSimulation(CoreSpec(grid=g, nu=nu, advection=scheme))
    u, v, w, th = taylor_green(g, amp=0.0)
    o.set_state(U * u, U * v, w, 0 * th)
    for _ in range(int(round(T / dt))):
        o.step_rk3(dt)
    return o


def test_rk3_third_order_in_time():
    g = regular_grid((16, 16, 16), (2 * np.pi,) * 3)
    nu = 0.05
    Kref = _tg(g, nu, 1 / 80).kinetic_energy()
    e1 = abs(_tg(g, nu, 0.1).kinetic_energy() - Kref)
    e2 = abs(_tg(g, nu, 0.05).kinetic_energy() - Kref)
    assert 6.5 < e1 / e2 < 9.5


def test_taylor_green_decays_at_the_discrete_rate():
    n, nu, U = 16, 0.05, 1e-3
    g = regular_grid((n, n, n), (2 * np.pi,) * 3)
    K0 = _tg(g, nu, 1.0, U=U, T=0.0).kinetic_energy()
    o = _tg(g, nu, 0.05, U=U, T=1.0)
    d = 2 * np.pi / n
    k2 = 3 * (2 / d * np.sin(d / 2)) ** 2
    assert abs(o.kinetic_energy() / K0 / np.exp(-2 * nu * k2) - 1) < 1e-4
    assert o.max_divergence() < 1e-12


@pytest.mark.parametrize("scheme", ["weno_js5", "weno_z5"])
def test_weno_taylor_green_matches_centred_at_small_amplitude(scheme):
    # at small amplitude advection is negligible, every scheme decays at the
    # viscous rate of the 7-point Laplacian
    n, nu, U = 16, 0.05, 1e-3
    g = regular_grid((n, n, n), (2 * np.pi,) * 3)
    K0 = _tg(g, nu, 1.0, U=U, T=0.0, scheme=scheme).kinetic_energy()
    o = _tg(g, nu, 0.05, U=U, T=0.5, scheme=scheme)
    d = 2 * np.pi / n
    k2 = 3 * (2 / d * np.sin(d / 2)) ** 2
    assert abs(o.kinetic_energy() / K0 / np.exp(-2 * nu * k2 * 0.5) - 1) < 1e-3


def _scalar_advection_error(n, scheme):
    # theta advected by a uniform flow u = 1 over one step: the WENO flux
    # divergence of sin(x) converges at the design order (test/advection.jl)
    g = regular_grid((n, 4, 4), (2 * np.pi, 1.0, 1.0))
    o = OracleSimulation(CoreSpec(grid=g, advection=scheme))
    u = g.zeros()
    u[g.interior] = 1.0
    th = g.zeros()
    x = g.xnodes("c")
    dx = 2 * np.pi / n
    # cell averages of sin(x): WENO reconstructs face values from averages
    th[g.interior] = ((np.cos(x - dx / 2) - np.cos(x + dx / 2)) / dx)[None, None, :]
    o.set_state(u, g.zeros(), g.zeros(), th)
    tt = o.tendencies()[3][g.interior][0, 0]
    # exact cell-average tendency of -d/dx sin(x): -(sin(x_e)-sin(x_w))/dx
    exact = -(np.sin(x + dx / 2) - np.sin(x - dx / 2)) / dx
    return np.abs(tt - exact).max()


@pytest.mark.parametrize("scheme,order", [("weno_z5", 4.8), ("weno_js5", 4.0)])
def test_weno_design_order(scheme, order):
    e = [_scalar_advection_error(n, scheme) for n in (32, 64)]
    assert np.log2(e[0] / e[1]) > order


# ---------------------------------------------------------------- anelastic -
def _cbl_spec(nz=16, c_s=0.17, flux=0.1):
    from aeolus_b200.grids import tanh_beta_for_first_cell
    lz = 2000.0
    beta = tanh_beta_for_first_cell(nz, lz, 8.0 * 128 / nz)
    g = stretched_grid((16, 16, nz), (640.0, 640.0, lz), tanh_faces(nz, lz, beta))
    from aeolus_b200.inputs import cbl_theta_profile
    th = cbl_theta_profile(g.znodes("c"))
    prof = anelastic_profiles(g, exponential_density(g), th)
    spec = CoreSpec(grid=g, core="anelastic", c_s=c_s, flux_bot=flux, wc=prof["wc"], wf=prof["wf"], thf=prof["thf"])
    return g, spec, th


def test_anelastic_rest_state_is_hydrostatic():
    g, spec, th = _cbl_spec(c_s=0.0, flux=0.0)
    o = OracleSimulation(spec)
    t = g.zeros()
    t[g.interior] = th[:, None, None]
    o.set_state(g.zeros(), g.zeros(), g.zeros(), t)
    o.step_rk3(1.0, 2)
    u, v, w, tt = o.get_state()
    assert np.abs(w[g.interior]).max() < 1e-12
    assert np.abs(tt[g.interior] - t[g.interior]).max() < 1e-10


def test_anelastic_constraint_at_round_off_after_steps():
    g, spec, th = _cbl_spec()
    o = OracleSimulation(spec)
    from aeolus_b200.inputs import cbl_initial
    u, v, w, t, _ = cbl_initial(g, seed=1, noise=0.1)
    o.set_state(u, v, w, t)
    o.step_rk3(1.0, 3)
    assert o.max_divergence() < 1e-13
    assert np.abs(o.get_field("w")[g.interior]).max() > 0  # the surface flux drives motion


# ---------------------------------------------------------------- adaptive dt
def test_adaptive_dt_advective_limit_growth_and_clamp():
    from aeolus_b200.simulation import CFLConstraints
    n = 16
    g = regular_grid((n, n, n), (2 * np.pi,) * 3)
    o = OracleSimulation(CoreSpec(grid=g, nu=0.0))
    rng = np.random.default_rng(1)
    st = []
    for name in ("u", "v", "w"):
        a = g.zeros()
        a[g.interior] = rng.standard_normal((n, n, n))
        o.set_field(name, a)
        st.append(a)
    o.fill_halos()
    u, v, w, _ = o.get_state()
    I = g.interior
    hz, hy, hx = g.halo[2], g.halo[1], g.halo[0]
    au = np.maximum(np.abs(u[I]), np.abs(u[hz:hz + n, hy:hy + n, hx + 1:hx + n + 1]))
    av = np.maximum(np.abs(v[I]), np.abs(v[hz:hz + n, hy + 1:hy + n + 1, hx:hx + n]))
    aw = np.maximum(np.abs(w[I]), np.abs(w[hz + 1:hz + n + 1, hy:hy + n, hx:hx + n]))
    rate = (au / g.dx + av / g.dy + aw / g.dz).max()
    dt, lim = o.adaptive_dt(CFLConstraints(C_advective=0.5))
    assert abs(dt - 0.5 / rate) <= 1e-14 * dt and lim == 0
    dt2, lim2 = o.adaptive_dt(CFLConstraints(), dt_prev=0.5 * dt)
    assert abs(dt2 - 1.1 * 0.5 * dt) <= 1e-15 and lim2 == 5
    dt3, lim3 = o.adaptive_dt(CFLConstraints(dt_max=0.1 * dt))
    assert dt3 == 0.1 * dt and lim3 == 7


def test_adaptive_dt_diffusive_limit_binds_for_viscous_flow():
    from aeolus_b200.simulation import CFLConstraints
    g = regular_grid((16, 16, 16), (1.0, 1.0, 1.0))
    o = OracleSimulation(CoreSpec(grid=g, nu=1.0))
    a = g.zeros()
    a[g.interior] = 1e-3
    o.set_field("u", a)
    dt, lim = o.adaptive_dt(CFLConstraints())
    harm = 1 / (3 / g.dx ** 2)
    assert lim == 1 and abs(dt - 0.25 * harm / 1.0) < 1e-15


def test_isotropic_field_is_real_with_the_target_rms_and_projects_to_round_off():
    from aeolus_b200.inputs import isotropic_turbulence
    g = regular_grid((32, 32, 32), (2 * np.pi,) * 3)
    u, v, w = isotropic_turbulence(g, 1.0, 4.0, seed=1)
    I = g.interior
    rms = [np.sqrt((a[I] ** 2).mean()) for a in (u, v, w)]
    assert all(0.8 < r < 1.2 for r in rms)
    o = OracleSimulation(CoreSpec(grid=g))
    o.set_state(u, v, w, g.zeros())
    assert o.max_divergence() > 1e-3          # the continuous field's discrete divergence
    o.project()
    assert o.max_divergence() < 1e-12
