"""The RK3 step with the multigrid-preconditioned CG projection (solver="pcg").

* Every face open: the projection solves the same discrete Poisson problem as
  the column solver (periodic x, y; Neumann walls in z), so steps agree with
  the column solver's to the CG tolerance (relative L2 <= 1e-8 per field at
  tol 1e-12).
* The heated urban step on the staircase geometry of boxes (0/1 apertures
  from a solid mask, the urban cases' obstacle model): 12 FP64 steps at
  dt = 1 s match the oracle to relative L2 <= 1e-9 per field; FP32-mixed
  (theta held as its deviation from theta0) stays within 1e-5 of FP64.
* Floor-standing boxes: FP64 steps match the oracle's cut-cell projection
  (the same multigrid-preconditioned CG on the CPU) to relative L2 <= 1e-10
  per field at tol 1e-12, centred and WENO-JS5 with Smagorinsky.
* Floor-standing boxes (cut-cell apertures): after every step each blocked
  face carries zero velocity and the aperture-weighted divergence is the
  solve's residual (max <= 1e-6 U/dx at tol 1e-10), the device diagnostic
  agrees with the host's; on staircase boxes FP32-mixed stays within 1e-5 of
  FP64; the learned U-Net preconditioner (untrained: the fallback to the
  cycle carries the solve) reaches the same tolerance.
"""
import numpy as np
import pytest

from aeolus_b200 import CoreSpec, regular_grid
from aeolus_b200.cutcell import (box_geometry, box_solid_mask, face_coefficients, random_boxes,
                                 staircase_geometry)

pytestmark = pytest.mark.gpu

FIELDS = ("u", "v", "w", "theta")
N = (32, 32, 16)
EXT = (64.0, 64.0, 32.0)


def Sim(spec):
    from aeolus_b200.simulation import Simulation
    return Simulation(spec)


def grid():
    return regular_grid(N, EXT, halo=(3, 3, 3), bc_z="wall")


def spec(g, solver, precision="fp64"):
    return CoreSpec(grid=g, nu=1e-3, theta0=300.0, flux_bot=0.05, solver=solver, precision=precision)


def state(g, seed, fluid=None):
    rng = np.random.default_rng(seed)
    nx, ny, nz = g.size
    th = np.full(g.storage_shape, 300.0)
    th[g.interior] += 0.1 * rng.standard_normal((nz, ny, nx))
    u, v = g.zeros(), g.zeros()
    u[g.interior] = 0.5 + 0.1 * rng.standard_normal((nz, ny, nx))
    v[g.interior] = 0.1 * rng.standard_normal((nz, ny, nx))
    if fluid is not None:
        u[g.interior] *= fluid
        v[g.interior] *= fluid
    return u, v, g.zeros(), th


def rel_l2(a, b, g):
    a, b = a[g.interior], b[g.interior]
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def boxes():
    g = grid()
    geom = box_geometry(g, random_boxes(g, 4, seed=2, footprint=(8.0, 16.0), height=(6.0, 20.0)), nsub=4)
    return g, geom, face_coefficients(geom, power=1)


def host_divergence(g, ap, u, v, w):
    """max |sum_faces +-a u / h| over the interior (storage arrays, halos filled)."""
    ax, ay, az = ap
    hx, hy, hz = g.halo
    nx, ny, nz = g.size
    K, J = slice(hz, hz + nz), slice(hy, hy + ny)
    d = ((ax[:, :, 1:] * u[K, J, hx + 1:hx + nx + 1] - ax[:, :, :-1] * u[K, J, hx:hx + nx]) / g.dx
         + (ay[:, 1:, :] * v[K, hy + 1:hy + ny + 1, hx:hx + nx] - ay[:, :-1, :] * v[K, J, hx:hx + nx]) / g.dy)
    azz = az.copy()
    azz[0] = 0.0
    azz[-1] = 0.0
    d += (azz[1:] * w[hz + 1:hz + nz + 1, J, hx:hx + nx] - azz[:-1] * w[K, J, hx:hx + nx]) / g.dz
    return float(np.abs(d).max())


def test_open_pcg_step_matches_the_column_solver():
    g = grid()
    col, pcg = Sim(spec(g, "column")), Sim(spec(g, "pcg"))
    pcg.set_pcg(None, tol=1e-12, maxit=500)
    st = state(g, 3)
    for s in (col, pcg):
        s.set_state(*st)
        s.project()
    col.step_rk3(0.2, 3)
    pcg.step_rk3(0.2, 3)
    errs = {n: rel_l2(pcg.get_field(n), col.get_field(n), g) for n in FIELDS}
    assert all(e <= 1e-8 for e in errs.values()), errs
    assert pcg.pcg_stats()["status"] == "converged"


@pytest.mark.parametrize("advection,c_s", [("centred", 0.0), ("weno_js5", 0.17)])
def test_pcg_step_with_boxes_matches_the_oracle(advection, c_s):
    from oracle.oracle import OracleSimulation
    g, geom, ap = boxes()
    fluid = (~geom.is_solid[g.interior]).astype(float)
    sp = CoreSpec(grid=g, nu=1e-3, theta0=300.0, flux_bot=0.05, solver="pcg", advection=advection, c_s=c_s)
    gpu, ora = Sim(sp), OracleSimulation(sp)
    st = state(g, 11, fluid)
    for s in (gpu, ora):
        s.set_pcg(ap, tol=1e-12, maxit=500)
        s.set_state(*st)
        s.project()
        s.step_rk3(0.2, 3)
    errs = {n: rel_l2(gpu.get_field(n), ora.get_field(n), g) for n in FIELDS}
    assert all(e <= 1e-10 for e in errs.values()), errs
    a, b = gpu.pcg_stats(), ora.pcg_stats()
    assert a["status"] == b["status"] == "converged"
    assert abs(a["iterations"] - b["iterations"]) <= 1, (a, b)


def test_heated_staircase_step_matches_the_oracle():
    from oracle.oracle import OracleSimulation
    g = grid()
    geom = staircase_geometry(g, box_solid_mask(g, random_boxes(g, 4, seed=2, footprint=(8.0, 16.0),
                                                                   height=(6.0, 20.0))))
    ap = face_coefficients(geom, power=1)
    nx, ny, nz = g.size
    th = np.full(g.storage_shape, 300.0)
    th[g.interior] += 0.1 * (2 * np.random.default_rng(1).random((nz, ny, nx)) - 1)
    z = g.zeros()

    def sp(prec):
        return CoreSpec(grid=g, advection="weno_js5", c_s=0.17, theta0=300.0, flux_bot=0.15, solver="pcg",
                        precision=prec)

    sims = [Sim(sp("fp64")), Sim(sp("fp32_mixed")), OracleSimulation(sp("fp64"))]
    for s in sims:
        s.set_pcg(ap, tol=1e-12, maxit=500)
        s.set_state(z, z, z, th)
        s.project()
        s.step_rk3(1.0, 12)
    g64, g32, ora = sims
    e64 = {n: rel_l2(g64.get_field(n), ora.get_field(n), g) for n in FIELDS}
    assert all(e <= 1e-9 for e in e64.values()), e64
    e32 = {n: rel_l2(g32.get_field(n), g64.get_field(n), g) for n in FIELDS}
    assert all(e <= 1e-5 for e in e32.values()), e32
    assert np.abs(g64.get_field("w")[g.interior]).max() < 0.1


def test_pcg_step_with_boxes_blocks_faces_and_is_divergence_free():
    g, geom, ap = boxes()
    fluid = (~geom.is_solid[g.interior]).astype(float)
    s = Sim(spec(g, "pcg"))
    s.set_pcg(ap, tol=1e-10, maxit=500)
    s.set_state(*state(g, 5, fluid))
    s.project()
    for _ in range(3):
        s.step_rk3(0.2, 1)
        st = s.pcg_stats()
        assert st["status"] == "converged" and st["relative_residual"] <= 1e-10, st
    u, v, w = (s.get_field(n) for n in ("u", "v", "w"))
    hx, hy, hz = g.halo
    nx, ny, nz = g.size
    K, J = slice(hz, hz + nz), slice(hy, hy + ny)
    ax, ay, az = ap
    assert np.all(u[K, J, hx:hx + nx][ax[:, :, :-1] == 0] == 0)
    assert np.all(v[K, hy:hy + ny, hx:hx + nx][ay[:, :-1, :] == 0] == 0)
    assert np.all(w[hz:hz + nz, J, hx:hx + nx][az[:-1] == 0] == 0)
    scale = 0.5 / g.dx
    dh = host_divergence(g, ap, u, v, w)
    dd = s.max_divergence()
    assert dh <= 1e-6 * scale and dd <= 1e-6 * scale, (dh, dd)
    assert abs(dh - dd) <= 1e-9 * scale + 1e-6 * dh


def test_pcg_fp32_mixed_close_to_fp64():
    # staircase boxes: with fractional apertures the plain divergence of the
    # projected velocity is not zero at cut cells, so the Cartesian transport
    # of theta depends on the offset FP32 stores theta at
    g = grid()
    geom = staircase_geometry(g, box_solid_mask(g, random_boxes(g, 4, seed=2, footprint=(8.0, 16.0),
                                                                   height=(6.0, 20.0))))
    ap = face_coefficients(geom, power=1)
    fluid = (~geom.is_solid[g.interior]).astype(float)
    sims = [Sim(spec(g, "pcg", p)) for p in ("fp64", "fp32_mixed")]
    st = state(g, 7, fluid)
    for s in sims:
        s.set_pcg(ap, tol=1e-10, maxit=500)
        s.set_state(*st)
        s.project()
        s.step_rk3(0.2, 3)
    errs = {n: rel_l2(sims[1].get_field(n), sims[0].get_field(n), g) for n in FIELDS}
    assert all(e <= 1e-5 for e in errs.values()), errs


def test_pcg_step_with_the_learned_preconditioner_reaches_the_tolerance():
    from aeolus_b200.unet import UNet
    nl = (128, 16, 8)   # a grid the U-Net's 128-cell tiles cover at every level
    g = regular_grid(nl, (256.0, 32.0, 16.0), halo=(3, 3, 3), bc_z="wall")
    geom = box_geometry(g, random_boxes(g, 6, seed=4, footprint=(6.0, 12.0), height=(4.0, 10.0)), nsub=4)
    ap = face_coefficients(geom, power=1)
    fluid = (~geom.is_solid[g.interior]).astype(np.float32)
    s = Sim(spec(g, "pcg"))
    s.set_pcg(ap, tol=1e-8, maxit=500)
    net = UNet(nl, seed=0)
    net.set_mask(fluid)
    net.set_out_scale(1.0)
    s.set_learned(net, 0.9)
    s.set_state(*state(g, 9, fluid.astype(float)))
    s.project()
    s.step_rk3(0.2, 2)
    st = s.pcg_stats()
    assert st["status"] == "converged" and st["relative_residual"] <= 1e-8, st
    s.set_learned(None)
    s.step_rk3(0.2, 1)
    assert s.pcg_stats()["status"] == "converged"
