"""Open lateral faces (src/boundary_conditions/open_boundary.jl).

CPU (host and oracle):
* the mass-flux correction restates the reference's own checks
  (test/open_boundaries.jl:28-57), with the wall top this build keeps: a
  prescribed imbalance u = 1 + 0.2 x / Lx on the faces has Q = 0.2 Ly Lz;
  :none records it and corrects nothing; :uniform removes it with
  delta = Q / (total open area); :outflow_only removes it from the outflow
  face and leaves the inflow face as given; a uniform wind needs none;
* the plane slabs hold the data at the storage points of the faces (the
  normal velocity's boundary face on a west face at interior index 0);
* the oracle's projection leaves the prescribed boundary-face velocity
  unchanged, makes the aperture-weighted divergence (with the boundary
  fluxes) the solve's residual, and a uniform wind through an open box with
  matching data stays uniform over steps (the stepped check the reference
  describes and cut from its suite, :1-10).
GPU (-m gpu): the CUDA step with open x, and open x and y, over floor-standing
boxes, with and without Smagorinsky (whose eddy viscosity takes the mirror
across open faces, as the reference's nu_t halo fill gives it), matches the
oracle (FP64, relative L2 <= 1e-10 per field after 3 steps at tol 1e-12;
FP32-mixed within 1e-5 of FP64, the paired FP32 sweep included), keeps the
boundary faces and the uniform wind."""
import numpy as np
import pytest

from aeolus_b200 import CoreSpec, regular_grid
from aeolus_b200.cutcell import box_geometry, box_solid_mask, face_coefficients, random_boxes, staircase_geometry
from aeolus_b200.open_boundary import FunctionBoundaryData, ProfileBoundaryData, open_boundary_conditions

LX, LY, LZ = 800.0, 600.0, 400.0
Q_IMB = 0.2 * LY * LZ
FIELDS = ("u", "v", "w", "theta")


def imb_data():
    return FunctionBoundaryData(u=lambda x, y, z, t: 1.0 + 0.2 * x / LX, v=0.0, w=0.0, theta=300.0)


def imb_grid():
    return regular_grid((16, 12, 8), (LX, LY, LZ), halo=(3, 3, 3), bc_z="wall")


def test_mass_flux_correction_removes_the_imbalance():
    g = imb_grid()
    o0 = open_boundary_conditions(g, imb_data(), x="open", y="open", correction="none")
    assert o0.ledger["Q"] == pytest.approx(Q_IMB, rel=1e-12)
    assert o0.ledger["residual"] == o0.ledger["Q"]            # nothing corrected
    o1 = open_boundary_conditions(g, imb_data(), x="open", y="open", correction="uniform")
    assert o1.ledger["Q"] == pytest.approx(Q_IMB, rel=1e-12)
    assert abs(o1.ledger["residual"]) < 1e-9 * Q_IMB
    # delta = Q / (the open area: west, east, south and north; the top is a wall)
    assert o1.ledger["delta"] == pytest.approx(Q_IMB / (2 * (LY * LZ + LX * LZ)), rel=1e-12)
    o2 = open_boundary_conditions(g, imb_data(), x="open", y="open", correction="outflow_only")
    assert abs(o2.ledger["residual"]) < 1e-9 * Q_IMB
    H = g.halo[0]
    west = o2.plane("u", "west").data
    assert np.allclose(west[H:H + g.nz, H:H + g.ny, H], 1.0, rtol=0, atol=1e-15)
    o3 = open_boundary_conditions(g, ProfileBoundaryData(u=5.0, v=2.0, w=0.0, theta=300.0), x="open", y="open")
    assert abs(o3.ledger["Q"]) < 1e-9 * 5.0 * LY * LZ and abs(o3.ledger["delta"]) < 1e-12


def test_planes_hold_the_data_at_the_storage_points():
    g = imb_grid()
    o = open_boundary_conditions(g, imb_data(), x="open", correction="none")
    H = g.halo[0]
    nx = g.nx
    west, east = o.plane("u", "west"), o.plane("u", "east")
    # u is staggered in x: storage index i sits at x0 + (i - H) dx
    xw = (np.arange(0, H + 1) - H) * g.dx
    xe = (np.arange(H + nx, nx + 2 * H) - H) * g.dx
    assert west.data.shape == (g.nz + 2 * H, g.ny + 2 * H, H + 1)
    assert np.allclose(west.data[4, 5, :], 1.0 + 0.2 * xw / LX, rtol=0, atol=1e-14)
    assert np.allclose(east.data[4, 5, :], 1.0 + 0.2 * xe / LX, rtol=0, atol=1e-14)
    th = o.plane("theta", "east")
    assert th.data.shape == (g.nz + 2 * H, g.ny + 2 * H, H) and np.all(th.data == 300.0)
    with pytest.raises(ValueError):
        open_boundary_conditions(g, ProfileBoundaryData(u=1.0), x="open")           # no theta data
    with pytest.raises(ValueError):
        open_boundary_conditions(g, imb_data(), x="open", outflow="sommerfeld")      # no such mode


# ---------------------------------------------------------------- steps

N = (32, 32, 16)
EXT = (64.0, 64.0, 32.0)


def box_case(seed=2, staircase=False):
    g = regular_grid(N, EXT, halo=(3, 3, 3), bc_z="wall")
    boxes = random_boxes(g, 4, seed=seed, footprint=(8.0, 16.0), height=(6.0, 20.0))
    geom = staircase_geometry(g, box_solid_mask(g, boxes)) if staircase else box_geometry(g, boxes, nsub=4)
    return g, geom, face_coefficients(geom, power=1)


def open_box(g, geom, ap, **kw):
    """The open faces over the boxes: solid points where a box touches a face
    (mark_open_boundary_solids!), the correction weighted by the faces' apertures."""
    return open_boundary_conditions(g, inflow(), solid=geom.is_solid, apertures=ap, **kw)


def inflow(z0=0.2):
    return ProfileBoundaryData(u=lambda z: 2.0 * np.log(max(z, z0) / z0) / np.log(10.0 / z0), v=0.3, w=0.0,
                               theta=lambda z: 300.0 + 0.003 * z)


def start_state(g, seed, fluid):
    rng = np.random.default_rng(seed)
    nx, ny, nz = g.size
    u, v, w = g.zeros(), g.zeros(), g.zeros()
    u[g.interior] = (1.5 + 0.2 * rng.standard_normal((nz, ny, nx))) * fluid
    v[g.interior] = 0.2 * rng.standard_normal((nz, ny, nx)) * fluid
    th = np.full(g.storage_shape, 300.0)
    th[g.interior] += 0.003 * g.znodes("c")[:, None, None] + 0.05 * rng.standard_normal((nz, ny, nx))
    return u, v, w, th


def spec(g, advection="centred", precision="fp64", c_s=0.0):
    return CoreSpec(grid=g, nu=1e-3, theta0=300.0, advection=advection, solver="pcg", precision=precision, c_s=c_s)


def open_divergence(g, ap, u, v, w):
    """max |sum over faces of (+-) a u / h|, the boundary faces' velocities from the storage arrays."""
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


def test_oracle_open_projection_keeps_the_faces_and_the_constraint():
    from oracle.oracle import OracleSimulation
    g, geom, ap = box_case()
    fluid = (~geom.is_solid[g.interior]).astype(float)
    obc = open_box(g, geom, ap, x="open", y="periodic")
    o = OracleSimulation(spec(g, c_s=0.17))
    o.set_pcg(ap, tol=1e-12, maxit=500)
    o.set_open_boundaries(obc)
    o.set_state(*start_state(g, 5, fluid))
    o.project()
    o.step_rk3(0.1, 2)
    assert o.pcg_stats()["status"] == "converged"
    o.fill_halos()
    u, v, w = (o.get_field(n) for n in ("u", "v", "w"))
    H = g.halo[0]
    # the prescribed boundary faces: west (interior 0) and east (first halo layer)
    bw = obc.plane("u", "west").data[H:H + g.nz, H:H + g.ny, H]
    be = obc.plane("u", "east").data[H:H + g.nz, H:H + g.ny, 0]
    assert np.array_equal(u[H:H + g.nz, H:H + g.ny, H], bw)
    assert np.array_equal(u[H:H + g.nz, H:H + g.ny, H + g.nx], be)
    assert open_divergence(g, ap, u, v, w) < 1e-9


def test_oracle_uniform_wind_through_an_open_box_stays_uniform():
    from oracle.oracle import OracleSimulation
    g = regular_grid((16, 16, 8), (32.0, 32.0, 16.0), halo=(3, 3, 3), bc_z="wall")
    data = ProfileBoundaryData(u=2.0, v=0.5, w=0.0, theta=300.0)
    obc = open_boundary_conditions(g, data, x="open", y="open")
    o = OracleSimulation(CoreSpec(grid=g, nu=0.0, theta0=300.0, advection="weno_js5", solver="pcg"))
    o.set_pcg(None, tol=1e-12, maxit=500)
    o.set_open_boundaries(obc)
    u, v = g.zeros() + 2.0, g.zeros() + 0.5
    o.set_state(u, v, g.zeros(), np.full(g.storage_shape, 300.0))
    o.step_rk3(0.2, 10)
    assert np.abs(o.get_field("u")[g.interior] - 2.0).max() < 1e-12
    assert np.abs(o.get_field("v")[g.interior] - 0.5).max() < 1e-12
    assert np.abs(o.get_field("w")[g.interior]).max() < 1e-12


# ---------------------------------------------------------------- the CUDA step


def rel_l2(a, b, g):
    a, b = a[g.interior], b[g.interior]
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.gpu
@pytest.mark.parametrize("y,advection,c_s", [("periodic", "centred", 0.0), ("open", "weno_js5", 0.0),
                                             ("open", "centred", 0.17), ("periodic", "weno_js5", 0.17)])
def test_open_step_matches_the_oracle(y, advection, c_s):
    # with Smagorinsky the eddy viscosity takes the mirror across the open faces
    from aeolus_b200.simulation import Simulation
    from oracle.oracle import OracleSimulation
    g, geom, ap = box_case()
    fluid = (~geom.is_solid[g.interior]).astype(float)
    obc = open_box(g, geom, ap, x="open", y=y)
    sp = spec(g, advection, c_s=c_s)
    gpu, ora = Simulation(sp), OracleSimulation(sp)
    st = start_state(g, 7, fluid)
    for s in (gpu, ora):
        s.set_pcg(ap, tol=1e-12, maxit=500)
        s.set_open_boundaries(obc)
        s.set_state(*st)
        s.project()
        s.step_rk3(0.1, 3)
    # the step leaves the state with its open faces filled (the boundary face
    # of u holds the data, as the next stage's fill writes it); the oracle
    # returns it as its correction left it, so fill it first
    ora.fill_halos()
    errs = {n: rel_l2(gpu.get_field(n), ora.get_field(n), g) for n in FIELDS}
    assert all(e <= 1e-10 for e in errs.values()), errs
    a, b = gpu.pcg_stats(), ora.pcg_stats()
    assert a["status"] == b["status"] == "converged"
    # the halos the step leaves: the planes on the open faces
    H = g.halo[0]
    u = gpu.get_field("u")
    assert np.allclose(u[H:H + g.nz, H:H + g.ny, H + g.nx], obc.plane("u", "east").data[H:H + g.nz, H:H + g.ny, 0],
                       rtol=0, atol=1e-14)
    assert open_divergence(g, ap, u, gpu.get_field("v"), gpu.get_field("w")) < 1e-9
    assert gpu.max_divergence() < 1e-9


@pytest.mark.gpu
@pytest.mark.parametrize("advection,c_s", [("weno_js5", 0.0), ("centred", 0.17)])
def test_open_step_fp32_mixed_close_to_fp64(advection, c_s):
    # FP32 centred with Smagorinsky runs the paired sweep
    from aeolus_b200.simulation import Simulation
    # staircase boxes: with fractional apertures the Cartesian transport of
    # theta depends on the offset FP32 stores it at (the PCG step's own test)
    g, geom, ap = box_case(3, staircase=True)
    fluid = (~geom.is_solid[g.interior]).astype(float)
    obc = open_box(g, geom, ap, x="open", y="open")
    st = start_state(g, 9, fluid)
    out = {}
    for prec in ("fp64", "fp32_mixed"):
        s = Simulation(spec(g, advection, prec, c_s))
        s.set_pcg(ap, tol=1e-10, maxit=500)
        s.set_open_boundaries(obc)
        s.set_state(*st)
        s.project()
        s.step_rk3(0.1, 5)
        out[prec] = s
    errs = {n: rel_l2(out["fp32_mixed"].get_field(n), out["fp64"].get_field(n), g) for n in FIELDS}
    assert all(e <= 1e-5 for e in errs.values()), errs


@pytest.mark.gpu
def test_open_step_keeps_a_uniform_wind_and_closes_again():
    from aeolus_b200.simulation import Simulation
    g = regular_grid((32, 32, 8), (64.0, 64.0, 16.0), halo=(3, 3, 3), bc_z="wall")
    obc = open_boundary_conditions(g, ProfileBoundaryData(u=2.0, v=0.5, w=0.0, theta=300.0), x="open", y="open")
    s = Simulation(CoreSpec(grid=g, nu=0.0, theta0=300.0, advection="weno_z5", solver="pcg"))
    s.set_pcg(None, tol=1e-12, maxit=500)
    s.set_open_boundaries(obc)
    s.set_state(g.zeros() + 2.0, g.zeros() + 0.5, g.zeros(), np.full(g.storage_shape, 300.0))
    s.step_rk3(0.2, 10)
    assert np.abs(s.get_field("u")[g.interior] - 2.0).max() < 1e-12
    assert np.abs(s.get_field("w")[g.interior]).max() < 1e-12
    s.set_open_boundaries(None)                  # periodic again
    s.step_rk3(0.2, 2)
    assert np.abs(s.get_field("u")[g.interior] - 2.0).max() < 1e-12


# ---------------------------------------------------------------- radiating outflow


def pulse_residual(sim_cls, outflow, advection="centred", steps=200):
    """A theta pulse carried by a uniform wind out through the east face
    (x open, y periodic): the fraction of its integral of theta'^2 left in
    the box after it should have left."""
    g = regular_grid((64, 8, 8), (64.0, 8.0, 8.0), halo=(3, 3, 3), bc_z="wall")
    obc = open_boundary_conditions(g, ProfileBoundaryData(u=1.0, v=0.0, w=0.0, theta=300.0), x="open",
                                   outflow={"east": outflow})
    s = sim_cls(CoreSpec(grid=g, nu=0.0, theta0=0.0, advection=advection, solver="pcg"))
    s.set_pcg(None, tol=1e-12, maxit=500)
    s.set_open_boundaries(obc)
    th = np.full(g.storage_shape, 300.0)
    th[g.interior] += np.exp(-((g.xnodes("c") - 40.0) / 4.0) ** 2)[None, None, :]
    s.set_state(g.zeros() + 1.0, g.zeros(), g.zeros(), th)
    e0 = np.sum((s.get_field("theta")[g.interior] - 300.0) ** 2)
    s.step_rk3(0.25, steps)
    return np.sum((s.get_field("theta")[g.interior] - 300.0) ** 2) / e0, s


def test_oracle_convective_outflow_lets_a_pulse_leave():
    # the reference's radiation check (N-open-c, src/boundary_conditions/outflow.jl:240-285):
    # with centred advection a Dirichlet outflow keeps the pulse, the
    # second-order upstream radiation lets it leave
    from oracle.oracle import OracleSimulation
    kept, _ = pulse_residual(OracleSimulation, "dirichlet")
    left, _ = pulse_residual(OracleSimulation, "convective")
    orl, _ = pulse_residual(OracleSimulation, "orlanski")
    assert kept > 0.9 and left < 1e-3 and orl < 1e-2, (kept, left, orl)


def test_oracle_convective_outflow_over_boxes_stays_compatible():
    # radiated outflow over boxes that touch the faces: the aperture-weighted
    # correction leaves no net flux the cut-cell divergence sees, so every
    # projection converges and the divergence is the solve's residual
    from oracle.oracle import OracleSimulation
    g, geom, ap = box_case()
    fluid = (~geom.is_solid[g.interior]).astype(float)
    obc = open_box(g, geom, ap, x="open", y="open", outflow={"east": "convective", "north": "convective"})
    o = OracleSimulation(spec(g, "weno_js5", c_s=0.17))
    o.set_pcg(ap, tol=1e-12, maxit=500)
    o.set_open_boundaries(obc)
    o.set_state(*start_state(g, 13, fluid))
    o.project()
    for _ in range(3):
        o.step_rk3(0.1, 1)
        assert o.pcg_stats()["status"] == "converged"
        led = o.open_ledger()
        assert abs(led["residual"]) < 1e-9 * max(abs(led["Q"]), 1.0)
    o.fill_halos()
    assert open_divergence(g, ap, *(o.get_field(n) for n in ("u", "v", "w"))) < 1e-9


def test_convective_outflow_options():
    g = imb_grid()
    o = open_boundary_conditions(g, imb_data(), x="open", y="open", outflow={"east": "convective"})
    assert list(o.radiating) == [0, 1, 0, 0]
    with pytest.raises(ValueError):
        open_boundary_conditions(g, imb_data(), x="open", outflow={"north": "convective"})   # y is periodic
    o2 = open_boundary_conditions(g, imb_data(), x="open", outflow={"east": "orlanski"})
    assert list(o2.radiating) == [0, 2, 0, 0]
    with pytest.raises(ValueError):
        open_boundary_conditions(g, imb_data(), x="open", outflow={"east": "sommerfeld"})


@pytest.mark.gpu
@pytest.mark.parametrize("y,outflow,c_s", [("open", {"east": "convective", "north": "convective"}, 0.0),
                                           ("periodic", {"east": "convective"}, 0.17),
                                           ("open", {"east": "convective"}, 0.17),
                                           ("open", {"east": "convective", "north": "convective"}, 0.17),
                                           ("open", {"east": "orlanski", "north": "convective"}, 0.0),
                                           ("periodic", {"east": "orlanski"}, 0.17)])
def test_convective_outflow_matches_the_oracle(y, outflow, c_s):
    # radiating outflow over boxes that touch the faces; the imbalance of the
    # data and the radiated points corrected before every projection; with a
    # closure the strain at the corners of two open faces reads v's south
    # boundary face beyond the x faces, which the south plane sets
    from aeolus_b200.simulation import Simulation
    from oracle.oracle import OracleSimulation
    g, geom, ap = box_case()
    fluid = (~geom.is_solid[g.interior]).astype(float)
    obc = open_box(g, geom, ap, x="open", y=y, outflow=outflow)
    sp = spec(g, "weno_js5", c_s=c_s)
    gpu, ora = Simulation(sp), OracleSimulation(sp)
    st = start_state(g, 13, fluid)
    for s in (gpu, ora):
        s.set_pcg(ap, tol=1e-12, maxit=500)
        s.set_open_boundaries(obc)
        s.set_state(*st)
        s.project()
        s.step_rk3(0.1, 4)
    ora.fill_halos()
    errs = {n: rel_l2(gpu.get_field(n), ora.get_field(n), g) for n in FIELDS}
    assert all(e <= 1e-10 for e in errs.values()), errs
    a, b = gpu.open_ledger(), ora.open_ledger()
    assert abs(a["delta"] - b["delta"]) <= 1e-10 * max(abs(b["delta"]), 1e-12) + 1e-14, (a, b)
    assert abs(a["residual"]) < 1e-9 * max(abs(a["Q"]), 1.0)


@pytest.mark.gpu
def test_convective_outflow_lets_a_pulse_leave_on_the_device():
    from aeolus_b200.simulation import Simulation
    from oracle.oracle import OracleSimulation
    for mode, bound in (("convective", 1e-3), ("orlanski", 1e-2)):
        left, s = pulse_residual(Simulation, mode)
        ref, o = pulse_residual(OracleSimulation, mode)
        assert left < bound and abs(left - ref) <= 1e-9, (mode, left, ref)


def open_restart(sim_cls, tmp_path, outflow, steps=12):
    """A run with open faces checkpointed half-way (the planes and the
    :orlanski history with the fields; open_boundary_checkpoint and
    restore_open_boundary_checkpoint!, open_boundary.jl:1282-1350) and
    restarted on a fresh domain with the same faces: the restarted steps and
    the uninterrupted ones, and the restart with the history dropped."""
    from aeolus_b200.checkpoint import checkpoint, read_checkpoint, restore
    g = regular_grid((64, 8, 8), (64.0, 8.0, 8.0), halo=(3, 3, 3), bc_z="wall")
    obc = open_boundary_conditions(g, ProfileBoundaryData(u=1.0, v=0.1, w=0.0, theta=300.0), x="open", y="open",
                                   outflow=outflow)

    def make():
        s = sim_cls(CoreSpec(grid=g, nu=1e-3, theta0=300.0, advection="weno_js5", solver="pcg"))
        s.set_pcg(None, tol=1e-12, maxit=500)
        s.set_open_boundaries(obc)
        return s

    a = make()
    th = np.full(g.storage_shape, 300.0)
    th[g.interior] += np.exp(-((g.xnodes("c") - 40.0) / 4.0) ** 2)[None, None, :]
    rng = np.random.default_rng(5)
    v = g.zeros()
    v[g.interior] = 0.1 + 0.05 * rng.standard_normal(v[g.interior].shape)
    a.set_state(g.zeros() + 1.0, v, g.zeros(), th)
    a.project()
    a.step_rk3(0.25, steps)
    path = checkpoint(a, str(tmp_path / "open.npz"), t=steps * 0.25)
    a.step_rk3(0.25, steps)
    b = make()
    restore(b, path)
    b.step_rk3(0.25, steps)
    same = all(np.array_equal(a.get_field(n)[g.interior], b.get_field(n)[g.interior]) for n in FIELDS + ("p",))
    # the planes at the rows the interior reads (the points in the halo rows
    # radiate from the fields' halos, which the restart refills from the planes)
    (xa, ya), (xb, yb) = a.open_planes(), b.open_planes()
    (hx, hy, hz), (nx, ny, nz) = g.halo, g.size
    same = same and np.array_equal(xa[:, :, hz:hz + nz, hy:hy + ny], xb[:, :, hz:hz + nz, hy:hy + ny])
    same = same and np.array_equal(ya[:, :, hz:hz + nz, :, hx:hx + nx], yb[:, :, hz:hz + nz, :, hx:hx + nx])
    payload = read_checkpoint(path)
    c = make()
    if "hist_x" in payload["open"]:
        payload["open"]["hist_set"] = 0.0
    else:
        payload["open"] = None
    if payload["open"] is None:
        with pytest.raises(ValueError):
            restore(c, payload)
        return same, None
    restore(c, payload)
    c.step_rk3(0.25, steps)
    return same, max(np.abs(a.get_field(n)[g.interior] - c.get_field(n)[g.interior]).max() for n in FIELDS)


@pytest.mark.parametrize("outflow", [{}, {"east": "orlanski", "north": "convective"}])
def test_oracle_restart_with_open_faces_continues_exactly(tmp_path, outflow):
    from oracle.oracle import OracleSimulation
    same, dropped = open_restart(OracleSimulation, tmp_path, outflow)
    assert same
    assert dropped is None or dropped > 1e-9, dropped   # without the history the first phase speed differs


@pytest.mark.gpu
@pytest.mark.parametrize("outflow", [{}, {"east": "orlanski", "north": "convective"}])
def test_restart_with_open_faces_continues_exactly(tmp_path, outflow):
    from aeolus_b200.simulation import Simulation
    same, dropped = open_restart(Simulation, tmp_path, outflow)
    assert same
    assert dropped is None or dropped > 1e-9, dropped


def radiating_domain(sim_cls):
    g = regular_grid((64, 8, 8), (64.0, 8.0, 8.0), halo=(3, 3, 3), bc_z="wall")
    obc = open_boundary_conditions(g, ProfileBoundaryData(u=1.0, v=0.1, w=0.0, theta=300.0), x="open", y="open",
                                   outflow={"east": "orlanski", "north": "convective"})
    s = sim_cls(CoreSpec(grid=g, nu=1e-3, theta0=300.0, advection="weno_js5", solver="pcg"))
    s.set_pcg(None, tol=1e-12, maxit=500)
    s.set_open_boundaries(obc)
    th = np.full(g.storage_shape, 300.0)
    th[g.interior] += np.exp(-((g.xnodes("c") - 40.0) / 4.0) ** 2)[None, None, :]
    rng = np.random.default_rng(5)
    v = g.zeros()
    v[g.interior] = 0.1 + 0.05 * rng.standard_normal(v[g.interior].shape)
    s.set_state(g.zeros() + 1.0, v, g.zeros(), th)
    s.project()
    return g, s


@pytest.mark.gpu
def test_adaptive_step_with_radiating_faces_matches_the_oracle_and_rewinds_a_retry():
    # step_adaptive! over a radiating open set: the CFL pick and the steps
    # match the oracle's; a step whose guard fails is retried from its start,
    # the plane buffers, the boundary faces and the Orlanski history included,
    # so a run that failed once continues exactly as one that never did
    from aeolus_b200._lib import NumericalFailure
    from aeolus_b200.simulation import CFLConstraints, Simulation
    from oracle.oracle import OracleSimulation
    g, s = radiating_domain(Simulation)
    _, o = radiating_domain(OracleSimulation)
    c = CFLConstraints(C_advective=0.5, growth_max=1.1)
    dts_o = o.step_adaptive(c, 4)
    dts, dp = [], None
    for _ in range(4):
        st = s.step_adaptive(c, 1, dp)
        dts.append(st["dt"])
        dp = st["dt"]
        assert st["retries"] == 0
    assert np.allclose(dts, dts_o, rtol=1e-11, atol=0), (dts, dts_o)
    o.fill_halos()
    errs = {n: rel_l2(s.get_field(n), o.get_field(n), g) for n in FIELDS}
    assert all(e <= 1e-10 for e in errs.values()), errs
    _, a = radiating_domain(Simulation)
    _, b = radiating_domain(Simulation)
    a.step_rk3(0.25, 3)
    b.step_rk3(0.25, 3)
    with pytest.raises(NumericalFailure):
        a.step_adaptive(CFLConstraints(max_velocity=1e-3, max_retries=2), 1)
    for x in (a, b):
        x.step_adaptive(c, 3, 0.25)
    for n in FIELDS + ("p",):
        assert np.array_equal(a.get_field(n)[g.interior], b.get_field(n)[g.interior]), n
    (xa, ya), (xb, yb) = a.open_planes(), b.open_planes()
    (hx, hy, hz), (nx, ny, nz) = g.halo, g.size
    assert np.array_equal(xa[:, :, hz:hz + nz, hy:hy + ny], xb[:, :, hz:hz + nz, hy:hy + ny])
    assert np.array_equal(ya[:, :, hz:hz + nz, :, hx:hx + nx], yb[:, :, hz:hz + nz, :, hx:hx + nx])
