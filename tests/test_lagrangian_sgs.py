"""Lagrangian dynamic Smagorinsky (LagrangianDynamicSmagorinsky,
src/operators/lagrangian_sgs.jl; Meneveau, Lund & Cabot 1996): the Germano
identity of the dynamic procedure (3 x 3 x 3 box test filter, width ratio 3)
averaged backwards along pathlines.  Once per accepted step (advance_sgs!,
:306-355) the memories relax toward the identity of the state after the
step,

    I_LM <- max(eps LM + (1 - eps) I_LM(x - u^n dt), 0),
    I_MM <- eps MM + (1 - eps) I_MM(x - u^n dt),

with trilinear upstream values (periodic x, y wrap; a z wall clamps),
eps = (dt/T) / (1 + dt/T), T = theta Delta (max(I_LM, 1e-8 I_MM) I_MM)^(-1/8)
of the upstream memories (:545-568); the first commit sets I_MM = MM,
I_LM = C0^2 MM.  The coefficient of a step is min(C0^2, cs_max^2) before the
first commit, then clip(I_LM / I_MM, 0, cs_max^2) of the committed memory
(sgs_viscosity!, :214-236); nu_t = C_s^2 Delta^2 |S| with Delta^2 =
(dx dy dz)^(2/3).

Oracle (CPU): each of these steps equals a numpy statement of it; a
restored memory (sgs_state / restore_sgs_state!, :372-381) continues the
run bit for bit.  GPU (`-m gpu`): steps match the oracle (FP64 1e-11 in the
state and the memories; FP32-mixed 1e-5 in the state), so does the adaptive
step, and a failed guard leaves the memory as committed.
"""
import numpy as np
import pytest

from aeolus_b200 import CoreSpec, regular_grid
from oracle.oracle import OracleSimulation
from test_dynamic_sgs import dynamic_numpy, grid, state

FIELDS = ("u", "v", "w", "theta")
CS_MAX = 0.5
TH0 = 300.0
C0 = 0.16


def spec(g, advection="centred", precision="fp64", c_s=CS_MAX, memory_time=None, lag_c0=C0):
    return CoreSpec(grid=g, c_s=c_s, sgs="lagrangian", theta0=TH0, advection=advection, precision=precision,
                    lag_c0=lag_c0, lag_memory_time=memory_time)


def relax_numpy(g, mem, LM, MM, dt, theta=1.5, memory_time=None):
    """_lagrangian_relax! / _upstream_n / _relax_pairs! on interior arrays:
    the memories after one commit from `mem` = (I_LM, I_MM, U, V, W)."""
    ilm, imm, U, V, W = mem
    nz, ny, nx = ilm.shape
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    x = (i + 1) - U * (dt / g.dx)
    y = (j + 1) - V * (dt / g.dy)
    z = (k + 1) - W * (dt / g.dz)
    per_z = g.bc_z != "wall"
    if not per_z:
        z = np.clip(z, 1, nz)
    x0, y0, z0 = np.floor(x).astype(int), np.floor(y).astype(int), np.floor(z).astype(int)
    fx, fy, fz = x - x0, y - y0, z - z0
    lm = np.zeros_like(ilm)
    mm = np.zeros_like(imm)
    for dk in (0, 1):
        for dj in (0, 1):
            for di in (0, 1):
                a = (x0 + di - 1) % nx
                b = (y0 + dj - 1) % ny
                c = (z0 + dk - 1) % nz if per_z else np.clip(z0 + dk, 1, nz) - 1
                wgt = (1 - fx if di == 0 else fx) * (1 - fy if dj == 0 else fy) * (1 - fz if dk == 0 else fz)
                lm = lm + wgt * ilm[c, b, a]
                mm = mm + wgt * imm[c, b, a]
    if memory_time is not None:
        eps = np.full_like(lm, (dt / memory_time) / (1 + dt / memory_time))
    else:
        delta = (g.dx * g.dy * g.dz) ** (1 / 3)
        pos = mm > 0
        base = np.where(pos, np.maximum(lm, 1e-8 * mm) * mm, 1.0)
        Tl = theta * delta * base ** (-1 / 8)
        eps = np.where(pos, (dt / Tl) / (1 + dt / Tl), 1.0)
    return np.maximum(eps * LM + (1 - eps) * lm, 0.0), eps * MM + (1 - eps) * mm


def identity(g, sim):
    """LM, MM, |S| and the cell-centred velocity of the sim's state (halos filled)."""
    sim.fill_halos() if hasattr(sim, "fill_halos") else None
    return dynamic_numpy(g, *(sim.get_field(n) for n in ("u", "v", "w")), CS_MAX, parts=True)


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def test_first_commit_and_the_initial_coefficient():
    g = grid()
    o = OracleSimulation(spec(g))
    o.set_state(*state(g))
    o.project()
    assert o.sgs_state()[5] is False
    o.tendencies()
    d2 = (g.dx * g.dy * g.dz) ** (2 / 3)
    _, _, ms, _ = identity(g, o)
    nut = o.get_field("nut")[g.interior]
    assert rel(nut, min(C0 ** 2, CS_MAX ** 2) * d2 * ms) <= 1e-13
    o.step_rk3(2e-3, 1)
    ilm, imm, U, V, W, init = o.sgs_state()
    LM, MM, ms, (Uc, Vc, Wc) = identity(g, o)
    assert init is True
    assert rel(imm, MM) <= 1e-13 and rel(ilm, C0 ** 2 * MM) <= 1e-13
    for a, b in ((U, Uc), (V, Vc), (W, Wc)):
        assert np.array_equal(a, b)
    # the next step's coefficient: the committed memory's ratio, C0^2 where MM > 0
    o.tendencies()
    nut = o.get_field("nut")[g.interior]
    cs2 = np.where(MM > 0, min(C0 ** 2, CS_MAX ** 2), 0.0)
    assert rel(nut, cs2 * d2 * ms) <= 1e-13


@pytest.mark.parametrize("bc_z,memory_time", [("wall", None), ("periodic", None), ("wall", 0.01)])
def test_relaxation_along_pathlines(bc_z, memory_time):
    g = grid(bc_z)
    o = OracleSimulation(spec(g, memory_time=memory_time))
    o.set_state(*state(g))
    o.project()
    dt = 2e-3
    o.step_rk3(dt, 2)
    before = o.sgs_state()
    o.step_rk3(dt, 1)
    after = o.sgs_state()
    LM, MM, ms, cell = identity(g, o)
    nlm, nmm = relax_numpy(g, before[:5], LM, MM, dt, memory_time=memory_time)
    assert rel(after[0], nlm) <= 1e-12 and rel(after[1], nmm) <= 1e-12
    assert np.count_nonzero(after[0]) > after[0].size // 2
    for a, b in zip(after[2:5], cell):
        assert np.array_equal(a, b)
    # the departure points moved: the relaxed memory is not the identity itself
    assert rel(after[1], MM) > 1e-3
    o.tendencies()
    d2 = (g.dx * g.dy * g.dz) ** (2 / 3)
    cs2 = np.where(nmm > 0, np.clip(nlm / np.where(nmm > 0, nmm, 1.0), 0.0, CS_MAX ** 2), 0.0)
    assert rel(o.get_field("nut")[g.interior], cs2 * d2 * ms) <= 1e-12


def test_a_restored_memory_continues_bit_for_bit():
    g = grid()
    a = OracleSimulation(spec(g))
    a.set_state(*state(g))
    a.project()
    a.step_rk3(2e-3, 2)
    fields = a.get_state()
    mem = a.sgs_state()
    a.step_rk3(2e-3, 2)
    b = OracleSimulation(spec(g))
    b.set_state(*fields)
    b.set_sgs_state(mem)
    b.step_rk3(2e-3, 2)
    for n in FIELDS:
        assert np.array_equal(a.get_field(n), b.get_field(n)), n
    for x, y in zip(a.sgs_state()[:5], b.sgs_state()[:5]):
        assert np.array_equal(x, y)


def test_lagrangian_spec_validation():
    from aeolus_b200 import stretched_grid, tanh_faces
    g = stretched_grid((16, 16, 16), (1.0, 1.0, 0.5), tanh_faces(16, 0.5, 1.5), halo=(3, 3, 3))
    with pytest.raises(ValueError):
        CoreSpec(grid=g, c_s=CS_MAX, sgs="lagrangian")
    with pytest.raises(ValueError):
        CoreSpec(grid=regular_grid((16, 16, 16), (1.0,) * 3, halo=(1, 1, 1)), c_s=CS_MAX, sgs="lagrangian")
    with pytest.raises(ValueError):
        spec(grid(), memory_time=0.0)
    with pytest.raises(ValueError):
        spec(grid(), lag_c0=-1.0)


@pytest.mark.gpu
@pytest.mark.parametrize("advection,bc_z,memory_time", [("centred", "wall", None), ("weno_js5", "wall", None),
                                                        ("centred", "periodic", None), ("centred", "wall", 0.01)])
def test_gpu_lagrangian_steps_match_the_oracle(advection, bc_z, memory_time):
    from aeolus_b200.simulation import Simulation
    g = grid(bc_z)
    st = state(g)
    kw = dict(advection=advection, memory_time=memory_time)
    sims = [OracleSimulation(spec(g, **kw)), Simulation(spec(g, **kw)), Simulation(spec(g, precision="fp32_mixed", **kw))]
    out, mems = [], []
    for s in sims:
        s.set_state(*st)
        s.project()
        s.step_rk3(2e-3, 4)
        f = {n: s.get_field(n)[g.interior] for n in FIELDS}
        f["theta"] = f["theta"] - TH0
        out.append(f)
        mems.append(s.sgs_state())
    ora, g64, g32 = out
    e64 = {n: np.linalg.norm(g64[n] - ora[n]) / np.linalg.norm(ora[n]) for n in FIELDS}
    assert all(e <= 1e-11 for e in e64.values()), e64
    e32 = {n: np.linalg.norm(g32[n] - g64[n]) / np.linalg.norm(g64[n]) for n in FIELDS}
    assert all(e <= 1e-5 for e in e32.values()), e32
    m64 = [np.linalg.norm(a - b) / np.linalg.norm(b) for a, b in zip(mems[1][:5], mems[0][:5])]
    assert all(e <= 1e-10 for e in m64), m64
    assert mems[1][5] is True and mems[2][5] is True
    # FP32 memories: the identity's L and M are differences of filtered products
    m32 = [np.linalg.norm(a - b) / np.linalg.norm(b) for a, b in zip(mems[2][:2], mems[1][:2])]
    assert all(e <= 1e-3 for e in m32), m32


@pytest.mark.gpu
def test_gpu_lagrangian_euler_steps_and_restored_memory():
    from aeolus_b200.simulation import Simulation
    g = grid()
    st = state(g)
    o, s = OracleSimulation(spec(g)), Simulation(spec(g))
    for x in (o, s):
        x.set_state(*st)
        x.project()
        x.step(1e-3, 3)
    for n in FIELDS:
        a, b = s.get_field(n)[g.interior], o.get_field(n)[g.interior]
        assert np.linalg.norm(a - b) / np.linalg.norm(b) <= 1e-11, n
    # the oracle's memory and state restored into a new device domain continue as the oracle does
    r = Simulation(spec(g))
    r.set_state(*o.get_state())
    r.set_sgs_state(o.sgs_state())
    for x in (o, r):
        x.step_rk3(2e-3, 2)
    for n in FIELDS:
        a, b = r.get_field(n)[g.interior], o.get_field(n)[g.interior]
        assert np.linalg.norm(a - b) / np.linalg.norm(b) <= 1e-11, n


@pytest.mark.gpu
def test_gpu_lagrangian_adaptive_steps_and_failed_guard():
    from aeolus_b200._lib import NumericalFailure
    from aeolus_b200.simulation import CFLConstraints, Simulation
    g = grid()
    sp = spec(g)
    s, o = Simulation(sp), OracleSimulation(sp)
    for x in (s, o):
        x.set_state(*state(g, amp=0.5))
        x.project()
    c = CFLConstraints(C_advective=0.5)
    dts_o = o.step_adaptive(c, 3)
    dts_g, dt_prev = [], None
    for _ in range(3):
        r = s.step_adaptive(c, 1, dt_prev)
        dts_g.append(r["dt"])
        dt_prev = r["dt"]
    assert np.allclose(dts_g, dts_o, rtol=1e-11, atol=0)
    for n in ("u", "v", "w"):
        a, b = s.get_field(n)[g.interior], o.get_field(n)[g.interior]
        assert np.linalg.norm(a - b) / np.linalg.norm(b) <= 1e-10, n
    mem = s.sgs_state()
    with pytest.raises(NumericalFailure):
        s.step_adaptive(CFLConstraints(C_advective=0.5, max_velocity=1e-6, max_retries=2), 1, dt_prev)
    for a, b in zip(mem[:5], s.sgs_state()[:5]):
        assert np.array_equal(a, b)
