"""The implicit immersed-boundary correction after every predictor
(implicit_ibm_correction!, src/IBM.jl:295-300, as the post_predictor! hook of
the step, src/Simulations.jl:624-628).

Oracle (CPU): an empty mask and tau -> infinity leave the step unchanged;
with tau = 0 a box's faces are zeroed before every projection, so the flow
through the box is a small fraction of the free stream.  GPU (`-m gpu`): the
FP64 step matches the oracle to relative L2 <= 1e-11 per field after 3 RK3
steps (tau = 0 and tau = 2 s, a box straddling the periodic seam, centred and
WENO-JS5); FP32-mixed stays within 1e-5 of FP64.
"""
import numpy as np
import pytest

from aeolus_b200 import CoreSpec, regular_grid
from oracle.oracle import OracleSimulation

FIELDS = ("u", "v", "w", "theta")


def grid():
    return regular_grid((32, 16, 16), (64.0, 32.0, 32.0), halo=(3, 3, 3), bc_z="wall")


def spec(g, advection="centred", precision="fp64"):
    return CoreSpec(grid=g, nu=1e-2, theta0=300.0, flux_bot=0.05, advection=advection, precision=precision,
                    solver="column")


def state(g, seed=3):
    rng = np.random.default_rng(seed)
    nx, ny, nz = g.size
    th = np.full(g.storage_shape, 300.0)
    th[g.interior] += 0.1 * rng.standard_normal((nz, ny, nx))
    u, v = g.zeros(), g.zeros()
    u[g.interior] = 1.0 + 0.1 * rng.standard_normal((nz, ny, nx))
    v[g.interior] = 0.1 * rng.standard_normal((nz, ny, nx))
    return u, v, g.zeros(), th


def mask(g):
    """A box over the periodic seam in x (cells 28..31 and 0..3), y 4..11, z 0..7."""
    m = np.zeros(g.storage_shape, dtype=np.uint8)
    hx, hy, hz = g.halo
    for i in list(range(28, 32)) + list(range(0, 4)):
        m[hz:hz + 8, hy + 4:hy + 12, hx + i] = 1
    return m


def run(sim, g, m=None, tau=0.0, steps=3):
    if m is not None:
        sim.set_ibm(m, tau)
    sim.set_state(*state(g))
    sim.project()
    sim.step_rk3(0.2, steps)
    return {n: sim.get_field(n)[g.interior] for n in FIELDS}


def test_empty_mask_and_infinite_tau_leave_the_step_unchanged():
    g = grid()
    ref = run(OracleSimulation(spec(g)), g)
    empty = run(OracleSimulation(spec(g)), g, np.zeros(g.storage_shape, np.uint8), 0.0)
    soft = run(OracleSimulation(spec(g)), g, mask(g), 1e300)
    for n in FIELDS:
        assert np.array_equal(empty[n], ref[n])
        assert np.array_equal(soft[n], ref[n])


def test_a_hard_box_blocks_the_flow():
    g = grid()
    m = mask(g)
    out = run(OracleSimulation(spec(g)), g, m, 0.0, steps=5)
    solid = m[g.interior].astype(bool)
    assert np.abs(out["u"][solid]).mean() < 0.2 * np.abs(out["u"][~solid]).mean()


def test_set_ibm_is_rejected_with_the_pcg_solver():
    g = grid()
    o = OracleSimulation(CoreSpec(grid=g, solver="pcg"))
    with pytest.raises(ValueError):
        o.set_ibm(mask(g), 0.0)


@pytest.mark.gpu
@pytest.mark.parametrize("advection,tau", [("centred", 0.0), ("weno_js5", 2.0)])
def test_gpu_matches_the_oracle(advection, tau):
    from aeolus_b200.simulation import Simulation
    g = grid()
    m = mask(g)
    ora = run(OracleSimulation(spec(g, advection)), g, m, tau)
    gpu = run(Simulation(spec(g, advection)), g, m, tau)
    errs = {n: np.linalg.norm(gpu[n] - ora[n]) / np.linalg.norm(ora[n]) for n in FIELDS}
    assert all(e <= 1e-11 for e in errs.values()), errs
    f32 = run(Simulation(spec(g, advection, "fp32_mixed")), g, m, tau)
    errs = {n: np.linalg.norm(f32[n] - gpu[n]) / np.linalg.norm(gpu[n]) for n in FIELDS}
    assert all(e <= 1e-5 for e in errs.values()), errs
