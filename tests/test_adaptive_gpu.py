"""Adaptive time stepping and the spectral isotropic initial field on the
GPU, against the oracle (decaying isotropic turbulence, WENO-Z5, no SGS).

  * the device field generator equals the host restatement of
    isotropic_turbulence_field! (src/operators/spectra.jl:312-343);
  * the on-device adaptive_dt pick equals the oracle's (src/TimeIntegration.jl:436-454);
  * adaptive SSP-RK3 steps give the same dt sequence and fields;
  * a step whose guard fails is retried with half the dt and, past the retry
    budget, raises NumericalFailure with the step-start state kept
    (src/TimeIntegration.jl:866-914).
"""
import numpy as np
import pytest

from aeolus_b200 import CoreSpec, regular_grid
from aeolus_b200.inputs import isotropic_turbulence
from oracle.oracle import OracleSimulation

pytestmark = pytest.mark.gpu


def Sim(spec):
    from aeolus_b200.simulation import Simulation
    return Simulation(spec)


def cfl(**kw):
    from aeolus_b200.simulation import CFLConstraints
    return CFLConstraints(**kw)


def hit_state(g, o):
    """Host field -> oracle, projected and scaled to u_rms = 1."""
    u, v, w = isotropic_turbulence(g, 1.0, 4.0, seed=1)
    o.set_state(u, v, w, g.zeros())
    o.project()
    u, v, w, _ = o.get_state()
    I = g.interior
    rms = np.sqrt((np.sum(u[I] ** 2) + np.sum(v[I] ** 2) + np.sum(w[I] ** 2)) / (3 * g.ncells))
    return tuple(a / rms for a in (u, v, w))


def test_device_isotropic_field_matches_the_host_generator():
    g = regular_grid((32, 16, 32), (2 * np.pi, np.pi, 2 * np.pi))
    s = Sim(CoreSpec(grid=g, advection="weno_z5"))
    s.init_isotropic(u_rms=1.0, k_peak=4.0, seed=7, project=False)
    ref = isotropic_turbulence(g, 1.0, 4.0, seed=7)
    for n, r in zip(("u", "v", "w"), ref):
        a = s.get_field(n)[g.interior]
        assert np.abs(a - r[g.interior]).max() <= 1e-12 * np.abs(r[g.interior]).max(), n


def test_device_projection_and_rescale_match_the_oracle():
    g = regular_grid((32, 32, 32), (2 * np.pi,) * 3)
    spec = CoreSpec(grid=g, advection="weno_z5")
    s, o = Sim(spec), OracleSimulation(spec)
    s.init_isotropic(u_rms=1.0, k_peak=4.0, seed=1, project=True, target_rms=1.0)
    ref = hit_state(g, o)
    for n, r in zip(("u", "v", "w"), ref):
        a = s.get_field(n)[g.interior]
        assert np.abs(a - r[g.interior]).max() <= 1e-12 * np.abs(r[g.interior]).max(), n
    assert s.max_divergence() < 1e-12


def test_adaptive_dt_pick_and_steps_match_the_oracle():
    g = regular_grid((32, 32, 32), (2 * np.pi,) * 3)
    spec = CoreSpec(grid=g, advection="weno_z5", nu=0.0)
    s, o = Sim(spec), OracleSimulation(spec)
    u, v, w = hit_state(g, o)
    for x in (s, o):
        x.set_state(u, v, w, g.zeros())
    c = cfl(C_advective=0.5, growth_max=1.1)
    d = s.cfl_diagnostics(c)
    dto, lim = o.adaptive_dt(c)
    assert abs(d["dt"] - dto) <= 1e-13 * dto and d["limiter"] == "advective" and lim == 0
    dts_o = o.step_adaptive(c, 6)
    dts_g = []
    dt_prev = None
    for _ in range(6):
        st = s.step_adaptive(c, 1, dt_prev)
        dts_g.append(st["dt"])
        dt_prev = st["dt"]
        assert st["retries"] == 0 and st["max_divergence"] < 1e-12
    assert np.allclose(dts_g, dts_o, rtol=1e-11, atol=0)
    for n in ("u", "v", "w"):
        a, b = s.get_field(n)[g.interior], o.get_field(n)[g.interior]
        assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-10, n


def test_failed_guard_retries_then_raises_with_the_start_state_kept():
    from aeolus_b200._lib import NumericalFailure
    g = regular_grid((16, 16, 16), (2 * np.pi,) * 3)
    spec = CoreSpec(grid=g, advection="weno_z5")
    s = Sim(spec)
    s.init_isotropic(u_rms=1.0, k_peak=4.0, seed=3, project=True, target_rms=1.0)
    before = [s.get_field(n) for n in ("u", "v", "w")]
    # a speed cap below the current speed: every attempt fails its guard
    with pytest.raises(NumericalFailure):
        s.step_adaptive(cfl(max_velocity=1e-3, max_retries=2), 1)
    after = [s.get_field(n) for n in ("u", "v", "w")]
    for a, b in zip(before, after):
        assert np.array_equal(a, b)
    # with a sane cap the same state steps normally
    st = s.step_adaptive(cfl(), 2)
    assert st["retries"] == 0 and st["t_advanced"] > 0
