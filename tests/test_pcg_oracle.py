"""The oracle's cut-cell projection (solver="pcg") on the CPU.

Restates the reference's cut-cell checks for the projection the stepping
engine uses with the multigrid-preconditioned CG:
  * L = D G: the a^2-weighted operator the CG inverts is the aperture
    divergence of the aperture gradient      test/cutcell.jl:59-87
  * no penetration: every blocked face carries zero velocity after a
    projection                                test/cutcell.jl:118-133
  * the projected velocity is divergence-free to the solve's residual
    (the urban smoke check, src/components/urban/pressure_solver.jl:126-131)
  * the staircase geometry of a solid mask has 0/1 fractions and apertures
    (cut_cell_geometry(mesh, ::SolidMask), src/CutCell.jl:334-352), and the
    heated urban step on it stays bounded (with fractional apertures the
    step's Cartesian transport is not conservative and theta runs away)
and ties the projection to the column solver, which solves the same discrete
Poisson problem when every face is open.
"""
import numpy as np
import pytest

from aeolus_b200 import CoreSpec, regular_grid
from aeolus_b200.cutcell import (box_geometry, box_solid_mask, face_coefficients, random_boxes,
                                 staircase_geometry)
from oracle.mgpcg import OracleMGPCG
from oracle.oracle import OracleSimulation

N = (32, 32, 16)
EXT = (64.0, 64.0, 32.0)
FIELDS = ("u", "v", "w", "theta")


def grid():
    return regular_grid(N, EXT, halo=(3, 3, 3), bc_z="wall")


def spec(g, solver, advection="centred"):
    return CoreSpec(grid=g, nu=1e-3, theta0=300.0, flux_bot=0.05, solver=solver, advection=advection)


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


def boxes(g):
    geom = box_geometry(g, random_boxes(g, 4, seed=2, footprint=(8.0, 16.0), height=(6.0, 20.0)), nsub=4)
    return geom, face_coefficients(geom, power=1)


@pytest.mark.parametrize("advection", ["centred", "weno_js5"])
def test_open_pcg_projection_equals_the_column_projection(advection):
    g = grid()
    col, pcg = OracleSimulation(spec(g, "column", advection)), OracleSimulation(spec(g, "pcg", advection))
    pcg.set_pcg(None, tol=1e-13, maxit=500)
    st = state(g, 3)
    for s in (col, pcg):
        s.set_state(*st)
        s.project()
        s.step_rk3(0.2, 3)
    for n in FIELDS:
        a, b = col.get_field(n)[g.interior], pcg.get_field(n)[g.interior]
        assert np.linalg.norm(a - b) <= 1e-12 * np.linalg.norm(a), n
    assert pcg.pcg_stats()["status"] == "converged"


def test_aperture_operator_is_divergence_of_gradient():
    """A phi = D(a G phi) with G phi = a d(phi)/h on every face and D the
    aperture-weighted divergence: the a^2 operator of the CG."""
    g = grid()
    geom, (ax, ay, az) = boxes(g)
    az = az.copy()
    az[0] = 0.0
    az[-1] = 0.0
    nx, ny, nz = g.size
    phi = np.random.default_rng(5).standard_normal((nz, ny, nx))
    gx = np.zeros((nz, ny, nx + 1))
    gx[:, :, 1:nx] = (phi[:, :, 1:] - phi[:, :, :-1]) / g.dx
    gx[:, :, 0] = gx[:, :, nx] = (phi[:, :, 0] - phi[:, :, -1]) / g.dx
    gy = np.zeros((nz, ny + 1, nx))
    gy[:, 1:ny, :] = (phi[:, 1:, :] - phi[:, :-1, :]) / g.dy
    gy[:, 0, :] = gy[:, ny, :] = (phi[:, 0, :] - phi[:, -1, :]) / g.dy
    gz = np.zeros((nz + 1, ny, nx))
    gz[1:nz] = (phi[1:] - phi[:-1]) / g.dz
    fx, fy, fz = ax * ax * gx, ay * ay * gy, az * az * gz
    dg = (fx[:, :, 1:] - fx[:, :, :-1]) / g.dx + (fy[:, 1:, :] - fy[:, :-1, :]) / g.dy + (fz[1:] - fz[:-1]) / g.dz
    op = OracleMGPCG(N, (g.dx, g.dy, g.dz), coeffs=(ax * ax, ay * ay, az * az)).apply(phi)
    assert np.abs(op - dg).max() <= 1e-12 * np.abs(dg).max()
    # negative semi-definite (test/cutcell.jl:85)
    assert float((phi * op).sum()) < 0


def test_pcg_projection_blocks_faces_and_is_divergence_free():
    g = grid()
    geom, ap = boxes(g)
    fluid = (~geom.is_solid[g.interior]).astype(float)
    s = OracleSimulation(spec(g, "pcg"))
    s.set_pcg(ap, tol=1e-10, maxit=500)
    s.set_state(*state(g, 5, fluid))
    s.project()
    s.step_rk3(0.2, 2)
    st = s.pcg_stats()
    assert st["status"] == "converged" and st["relative_residual"] <= 1e-10, st
    hx, hy, hz = g.halo
    nx, ny, nz = g.size
    K, J = slice(hz, hz + nz), slice(hy, hy + ny)
    ax, ay, az = ap
    u, v, w = (s.get_field(n) for n in ("u", "v", "w"))
    assert np.all(u[K, J, hx:hx + nx][ax[:, :, :-1] == 0] == 0)
    assert np.all(v[K, hy:hy + ny, hx:hx + nx][ay[:, :-1, :] == 0] == 0)
    assert np.all(w[hz:hz + nz, J, hx:hx + nx][az[:-1] == 0] == 0)
    assert s.max_divergence() <= 1e-6 * 0.5 / g.dx


def test_pcg_solver_rejects_what_it_does_not_define():
    g = grid()
    s = OracleSimulation(spec(g, "pcg"))
    nx, ny, nz = g.size
    bad = (np.full((nz, ny, nx + 1), 1.5), np.ones((nz, ny + 1, nx)), np.ones((nz + 1, ny, nx)))
    with pytest.raises(ValueError):
        s.set_pcg(bad)
    with pytest.raises(ValueError):
        s.set_pcg(None, tol=0.0)


def test_staircase_geometry_of_boxes():
    g = grid()
    bx = random_boxes(g, 4, seed=2, footprint=(8.0, 16.0), height=(6.0, 20.0))
    mask = box_solid_mask(g, bx)
    geom = staircase_geometry(g, mask)
    assert set(np.unique(geom.vol_frac)) <= {0.0, 1.0}
    for a in (geom.ax, geom.ay, geom.az):
        assert set(np.unique(a)) <= {0.0, 1.0}
    fl = ~geom.is_solid
    assert np.array_equal(geom.is_solid[g.interior], mask[g.interior])
    # a face is open iff both of its cells are fluid (away from the low-side storage faces)
    assert np.array_equal(geom.ax[:, :, 1:] > 0, fl[:, :, :-1] & fl[:, :, 1:])
    assert np.array_equal(geom.az[1:] > 0, fl[:-1] & fl[1:])
    # the box cells: a centre below the top inside the footprint is solid
    x0, x1, y0, y1, _, z1 = bx[0]
    hx, hy, hz = g.halo
    i = int((0.5 * (x0 + x1) - g.origin[0]) // g.dx) % g.nx
    j = int((0.5 * (y0 + y1) - g.origin[1]) // g.dy) % g.ny
    assert mask[hz, hy + j, hx + i]
    # the periodic halos hold the interior's images
    assert np.array_equal(mask[:, :, :hx], mask[:, :, g.nx:g.nx + hx])
    assert np.array_equal(mask[:, :hy, :], mask[:, g.ny:g.ny + hy, :])


def test_heated_staircase_step_stays_bounded():
    g = grid()
    geom = staircase_geometry(g, box_solid_mask(g, random_boxes(g, 4, seed=2, footprint=(8.0, 16.0),
                                                                   height=(6.0, 20.0))))
    ap = face_coefficients(geom, power=1)
    s = OracleSimulation(CoreSpec(grid=g, advection="weno_js5", c_s=0.17, theta0=300.0, flux_bot=0.15,
                                  solver="pcg"))
    s.set_pcg(ap, tol=1e-8, maxit=500)
    nx, ny, nz = g.size
    th = np.full(g.storage_shape, 300.0)
    th[g.interior] += 0.1 * (2 * np.random.default_rng(1).random((nz, ny, nx)) - 1)
    z = g.zeros()
    s.set_state(z, z, z, th)
    s.project()
    s.step_rk3(1.0, 12)
    w, t = s.get_field("w")[g.interior], s.get_field("theta")[g.interior]
    # buoyant growth from 0.1 K noise and 0.075 K/s of surface heating over 12 s
    assert np.abs(w).max() < 0.1
    assert t.min() > 299.8 and t.max() < 300.1 + 12 * 0.15 / g.dz + 0.1
    assert s.max_divergence() <= 1e-6 * 0.1 / g.dx
