"""The Deardorff (1980) prognostic-TKE closure with Moeng's (1984)
coefficients (TKEClosure, src/PrognosticSGS.jl): nu_t = c_k l sqrt(e),
kappa_t = (1 + 2l/Delta) nu_t, l = min(Delta, c_l sqrt(e)/N) where N^2 > 0
(tke_length_scale :93-110), c_k passed as c_s.  Once per accepted step
(advance_sgs!, :978-1002) e is transported (flux-limited WENO-Z5,
advect_positive!, plus div(2 nu_t grad e)), produced (P_s = nu_t D with D the
discrete dual of the momentum operator, dual_strain! :488-806; P_b =
-kappa_t N^2; a surface heat flux adds (g/theta0) F/2 to the wall levels) and
dissipated (c_eps = c_eps0 + c_eps1 l/Delta; linearised implicit or exact,
_tke_update_body :1077-1145).

Oracle (CPU): nu_t and kappa_t equal a numpy statement; the commit equals a
numpy statement built on an independent scatter form of D (each flux share
added to its cells, then the halo fold), for walls and periodic z, stable
and unstable N^2, the surface flux and both dissipation forms; D of a linear
shear is S^2.  GPU (`-m gpu`): steps match the oracle (FP64 1e-11 in the
state and e; FP32-mixed 1e-5 in the state, 1e-4 in e), Euler steps, the
adaptive step and a restored e.
"""
import numpy as np
import pytest

from aeolus_b200 import CoreSpec, regular_grid
from oracle.oracle import OracleSimulation

FIELDS = ("u", "v", "w", "theta")
CK = 0.1
TH0 = 300.0


def grid(bc_z="wall", n=(16, 16, 16)):
    return regular_grid(n, (1.0, 1.0, 0.5), halo=(3, 3, 3), bc_z=bc_z)


def spec(g, precision="fp64", advection="centred", dissipation="semi_implicit", flux_bot=0.0, **kw):
    return CoreSpec(grid=g, c_s=CK, sgs="tke", theta0=TH0, advection=advection, precision=precision,
                    tke_dissipation=dissipation, flux_bot=flux_bot, nu=1e-5, **kw)


def state(g, seed=11, amp=0.5, strat=2.0):
    """a stably stratified column (dtheta/dz = strat) with noise: N^2 of both signs"""
    rng = np.random.default_rng(seed)
    nx, ny, nz = g.size
    z = g.znodes("c")[:, None, None]
    th = np.full(g.storage_shape, TH0)
    th[g.interior] += strat * z + 0.05 * rng.standard_normal((nz, ny, nx))
    u, v, w = g.zeros(), g.zeros(), g.zeros()
    for a in (u, v, w):
        a[g.interior] = amp * rng.standard_normal((nz, ny, nx))
    if g.bc_z == "wall":
        w[g.halo[2]] = 0.0
    e = 1e-5 + 0.03 * rng.random((nz, ny, nx)) ** 2    # small e where N^2 > 0 limits l
    return (u, v, w, th), e


def pad_c(g, a):
    """a cell-centred interior array with halos: periodic x, y; z periodic or mirrored at walls"""
    hx, hy, hz = g.halo
    a = np.pad(a, ((0, 0), (hy, hy), (hx, hx)), mode="wrap")
    return np.pad(a, ((hz, hz), (0, 0), (0, 0)), mode="symmetric" if g.bc_z == "wall" else "wrap")


def n2_numpy(g, th):
    hz = g.halo[2]
    c = th[:, g.interior[1], g.interior[2]]
    lo, mid, hi = c[hz - 1:-hz - 1], c[hz:-hz], c[hz + 1:c.shape[0] - hz + 1]
    return (9.81 / TH0) * ((0.5 * (mid + hi)) - (0.5 * (lo + mid))) * (1 / g.dz)


def length_numpy(g, e, N2, c_l=0.76):
    delta = (g.dx * g.dy * g.dz) ** (1 / 3)
    sq = np.sqrt(np.maximum(e, 0))
    N = np.sqrt(np.maximum(N2, 0))
    stable = N2 > 0
    with np.errstate(divide="ignore", invalid="ignore"):
        l = np.where(stable, np.minimum(delta, c_l * sq / np.where(stable, N, 1.0)), delta)
        s = np.where(stable, np.maximum(sq / delta, N / c_l), sq / delta)
    return l, s, delta


def dual_numpy(g, u, v, w):
    """D by the scatter (each flux share of the momentum operator added to the
    cells of its nu, then the halo fold), the form dual_strain! replaced"""
    hx, hy, hz = g.halo
    nx, ny, nz = g.size
    ix2, iy2, iz2 = 1 / g.dx ** 2, 1 / g.dy ** 2, 1 / g.dz ** 2
    D = np.zeros((nz + 2, ny + 2, nx + 2))      # the interior plus one halo layer, index + 1

    def at(a, dk, dj, di):
        return a[hz + dk:hz + nz + dk, hy + dj:hy + ny + dj, hx + di:hx + nx + di]

    def add(share, cells):
        for (dk, dj, di) in cells:
            D[1 + dk:1 + dk + nz, 1 + dj:1 + dj + ny, 1 + di:1 + di + nx] += share

    p = at(u, 0, 0, 0)
    add(-p * (at(u, 0, 0, 1) - p) * ix2, [(0, 0, 0)])
    add(p * (p - at(u, 0, 0, -1)) * ix2, [(0, 0, -1)])
    add(0.25 * (-p * (at(u, 0, 1, 0) - p) * iy2), [(0, 0, -1), (0, 0, 0), (0, 1, -1), (0, 1, 0)])
    add(0.25 * (p * (p - at(u, 0, -1, 0)) * iy2), [(0, -1, -1), (0, -1, 0), (0, 0, -1), (0, 0, 0)])
    add(0.25 * (-p * (at(u, 1, 0, 0) - p) * iz2), [(0, 0, -1), (0, 0, 0), (1, 0, -1), (1, 0, 0)])
    add(0.25 * (p * (p - at(u, -1, 0, 0)) * iz2), [(-1, 0, -1), (-1, 0, 0), (0, 0, -1), (0, 0, 0)])
    p = at(v, 0, 0, 0)
    add(-p * (at(v, 0, 1, 0) - p) * iy2, [(0, 0, 0)])
    add(p * (p - at(v, 0, -1, 0)) * iy2, [(0, -1, 0)])
    add(0.25 * (-p * (at(v, 0, 0, 1) - p) * ix2), [(0, -1, 0), (0, 0, 0), (0, -1, 1), (0, 0, 1)])
    add(0.25 * (p * (p - at(v, 0, 0, -1)) * ix2), [(0, -1, -1), (0, 0, -1), (0, -1, 0), (0, 0, 0)])
    add(0.25 * (-p * (at(v, 1, 0, 0) - p) * iz2), [(0, -1, 0), (0, 0, 0), (1, -1, 0), (1, 0, 0)])
    add(0.25 * (p * (p - at(v, -1, 0, 0)) * iz2), [(-1, -1, 0), (-1, 0, 0), (0, -1, 0), (0, 0, 0)])
    p = at(w, 0, 0, 0)
    add(-p * (at(w, 1, 0, 0) - p) * iz2, [(0, 0, 0)])
    add(p * (p - at(w, -1, 0, 0)) * iz2, [(-1, 0, 0)])
    add(0.25 * (-p * (at(w, 0, 0, 1) - p) * ix2), [(-1, 0, 0), (0, 0, 0), (-1, 0, 1), (0, 0, 1)])
    add(0.25 * (p * (p - at(w, 0, 0, -1)) * ix2), [(-1, 0, -1), (0, 0, -1), (-1, 0, 0), (0, 0, 0)])
    add(0.25 * (-p * (at(w, 0, 1, 0) - p) * iy2), [(-1, 0, 0), (0, 0, 0), (-1, 1, 0), (0, 1, 0)])
    add(0.25 * (p * (p - at(w, 0, -1, 0)) * iy2), [(-1, -1, 0), (0, -1, 0), (-1, 0, 0), (0, 0, 0)])
    # the fold: x, then y, then z (periodic image, or the mirror at a wall)
    D[:, :, nx] += D[:, :, 0]; D[:, :, 1] += D[:, :, nx + 1]
    D[:, ny, :] += D[:, 0, :]; D[:, 1, :] += D[:, ny + 1, :]
    if g.bc_z == "wall":
        D[1] += D[0]; D[nz] += D[nz + 1]
    else:
        D[nz] += D[0]; D[1] += D[nz + 1]
    return D[1:-1, 1:-1, 1:-1]


def commit_numpy(g, o, fields, e_n, dt, exact=False, flux_bot=0.0, c_eps0=0.19, c_eps1=0.51):
    """advance_sgs! of the TKE closure from e^n and the state after the step"""
    u, v, w, th = fields
    N2 = n2_numpy(g, th)
    l, s, delta = length_numpy(g, e_n, N2)
    nu = CK * l * np.sqrt(np.maximum(e_n, 0))
    K2, E = pad_c(g, 2 * nu), pad_c(g, e_n)
    tr = o.advect_positive(u, v, w, E, dt, accumulate=False)[g.interior]
    hx, hy, hz = g.halo
    nx, ny, nz = g.size

    def sh(a, dk, dj, di):
        return a[hz + dk:hz + nz + dk, hy + dj:hy + ny + dj, hx + di:hx + nx + di]
    idx, idy, idz = 1 / g.dx, 1 / g.dy, 1 / g.dz
    f = {}
    for name, (dk, dj, di), ih in (("x", (0, 0, 1), idx), ("y", (0, 1, 0), idy), ("z", (1, 0, 0), idz)):
        kp = 0.5 * (sh(K2, 0, 0, 0) + sh(K2, dk, dj, di))
        km = 0.5 * (sh(K2, -dk, -dj, -di) + sh(K2, 0, 0, 0))
        f[name] = ((kp * (sh(E, dk, dj, di) - sh(E, 0, 0, 0)) * ih) - (km * (sh(E, 0, 0, 0) - sh(E, -dk, -dj, -di)) * ih)) * ih
    tr = tr + 1.0 * ((f["x"] + f["y"]) + f["z"])
    ce = 0.19 + 0.51 * l / delta if (c_eps0, c_eps1) == (0.19, 0.51) else c_eps0 + c_eps1 * l / delta
    Ps = nu * dual_numpy(g, u, v, w)
    kv = (1 + 2 * l / delta) * nu
    Psf = np.zeros_like(e_n)
    Psf[0] += 9.81 / TH0 * flux_bot / 2
    src = Ps + np.where(N2 < 0, -kv * N2, 0.0) + np.maximum(Psf, 0)
    with np.errstate(divide="ignore", invalid="ignore"):
        rb = np.where((N2 > 0) & (s > 0), (1 + 2 * l / delta) * CK * N2 / np.where(s > 0, s, 1.0), 0.0)
    rb = rb + np.where(Psf < 0, -Psf / np.maximum(e_n, np.finfo(float).tiny), 0.0)
    es = np.maximum(e_n + dt * (tr + src), 0.0)
    en = es / (1 + dt * (ce * s + rb))
    if exact:
        ok = (l > 0) & (es > 0)
        with np.errstate(divide="ignore"):
            e1 = (1 / (1 / np.sqrt(es) + ce * dt / (2 * l))) ** 2
        en = np.where(ok, e1 / (1 + dt * rb), en)
    return en


def rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def test_coefficients_are_deardorff_moeng():
    g = grid()
    o = OracleSimulation(spec(g))
    flds, e = state(g)
    o.set_state(*flds)
    o.set_sgs_state(e)
    o.fill_halos()
    o.tendencies()
    N2 = n2_numpy(g, o.get_field("theta"))
    assert (N2 > 0).any() and (N2 < 0).any()
    l, s, delta = length_numpy(g, e, N2)
    nu = CK * l * np.sqrt(e)
    assert rel(o.get_field("nut")[g.interior], nu) <= 1e-13
    assert rel(o.get_field("kt")[g.interior], (1 + 2 * l / delta) * nu) <= 1e-13
    assert (l < delta).any()      # the stability limit binds somewhere


def test_dual_strain_of_a_linear_shear_is_s_squared():
    g = grid("periodic")
    u, v, w = g.zeros(), g.zeros(), g.zeros()
    S = 0.7
    y = (np.arange(-g.halo[1], g.ny + g.halo[1]) + 0.5) * g.dy
    u[:] = S * y[None, :, None]
    D = dual_numpy(g, u, v, w)
    assert np.allclose(D[:, 2:-2, :], S ** 2, rtol=1e-12)


@pytest.mark.parametrize("bc_z,dissipation,flux_bot", [("wall", "semi_implicit", 0.0), ("wall", "exact", 0.05),
                                                        ("periodic", "semi_implicit", 0.0), ("wall", "semi_implicit", -0.05)])
def test_commit_is_the_tke_equation(bc_z, dissipation, flux_bot):
    g = grid(bc_z)
    sp = spec(g, dissipation=dissipation, flux_bot=flux_bot)
    o, helper = OracleSimulation(sp), OracleSimulation(sp)
    flds, e = state(g)
    o.set_state(*flds)
    o.set_sgs_state(e)
    o.project()
    dt = 2e-3
    o.step_rk3(dt, 1)
    e1 = o.sgs_state()
    after = tuple(o.get_field(n) for n in FIELDS)
    ref = commit_numpy(g, helper, after, e, dt, exact=dissipation == "exact", flux_bot=flux_bot)
    assert rel(e1, ref) <= 1e-12
    assert np.all(e1 >= 0) and rel(e1, e) > 1e-3


def test_tke_restart_and_validation():
    g = grid()
    flds, e = state(g)
    a = OracleSimulation(spec(g))
    a.set_state(*flds)
    a.set_sgs_state(e)
    a.step_rk3(2e-3, 2)
    mid, em = a.get_state(), a.sgs_state()
    a.step_rk3(2e-3, 2)
    b = OracleSimulation(spec(g))
    b.set_state(*mid)
    b.set_sgs_state(em)
    b.step_rk3(2e-3, 2)
    assert np.array_equal(a.sgs_state(), b.sgs_state())
    for n in FIELDS:
        assert np.array_equal(a.get_field(n), b.get_field(n))
    with pytest.raises(ValueError):
        spec(regular_grid((8, 8, 8), (1.0,) * 3, halo=(2, 2, 2)))
    with pytest.raises(ValueError):
        spec(g, dissipation="implicit")
    assert OracleSimulation(spec(g, tke_e0=0.03)).sgs_state().min() == 0.03


@pytest.mark.gpu
@pytest.mark.parametrize("bc_z,dissipation,advection,flux_bot", [("wall", "semi_implicit", "centred", 0.05),
                                                                  ("wall", "exact", "weno_z5", 0.0),
                                                                  ("periodic", "semi_implicit", "centred", 0.0)])
def test_gpu_tke_steps_match_the_oracle(bc_z, dissipation, advection, flux_bot):
    from aeolus_b200.simulation import Simulation
    g = grid(bc_z)
    flds, e = state(g)
    kw = dict(dissipation=dissipation, advection=advection, flux_bot=flux_bot)
    sims = [OracleSimulation(spec(g, **kw)), Simulation(spec(g, **kw)), Simulation(spec(g, precision="fp32_mixed", **kw))]
    out, es = [], []
    for s in sims:
        s.set_state(*flds)
        s.set_sgs_state(e)
        s.project()
        s.step_rk3(2e-3, 4)
        f = {n: s.get_field(n)[g.interior] for n in FIELDS}
        f["theta"] = f["theta"] - TH0
        out.append(f)
        es.append(s.sgs_state())
    ora, g64, g32 = out
    e64 = {n: np.linalg.norm(g64[n] - ora[n]) / np.linalg.norm(ora[n]) for n in FIELDS}
    assert all(x <= 1e-11 for x in e64.values()), e64
    assert np.linalg.norm(es[1] - es[0]) / np.linalg.norm(es[0]) <= 1e-11
    e32 = {n: np.linalg.norm(g32[n] - g64[n]) / np.linalg.norm(g64[n]) for n in FIELDS}
    assert all(x <= 1e-5 for x in e32.values()), e32
    assert np.linalg.norm(es[2] - es[1]) / np.linalg.norm(es[1]) <= 1e-4
    # the nu_t diagnostic of the device is the closure's
    nut = sims[1].get_field("nut")[g.interior]
    th = sims[1].get_field("theta")
    l, _, _ = length_numpy(g, es[1], n2_numpy(g, th))
    assert rel(nut, CK * l * np.sqrt(es[1])) <= 1e-12


@pytest.mark.gpu
def test_gpu_tke_euler_adaptive_and_restore():
    from aeolus_b200.simulation import CFLConstraints, Simulation
    g = grid()
    flds, e = state(g)
    o, s = OracleSimulation(spec(g)), Simulation(spec(g))
    for x in (o, s):
        x.set_state(*flds)
        x.set_sgs_state(e)
        x.project()
        x.step(1e-3, 2)
    assert np.linalg.norm(s.sgs_state() - o.sgs_state()) / np.linalg.norm(o.sgs_state()) <= 1e-11
    c = CFLConstraints(C_advective=0.5, C_diffusive=0.25)
    dts_o = o.step_adaptive(c, 3)
    dts_g, dt_prev = [], None
    for _ in range(3):
        r = s.step_adaptive(c, 1, dt_prev)
        dts_g.append(r["dt"])
        dt_prev = r["dt"]
    assert np.allclose(dts_g, dts_o, rtol=1e-11, atol=0)
    assert np.linalg.norm(s.sgs_state() - o.sgs_state()) / np.linalg.norm(o.sgs_state()) <= 1e-10
    r = Simulation(spec(g))
    r.set_state(*o.get_state())
    r.set_sgs_state(o.sgs_state())
    for x in (o, r):
        x.step_rk3(2e-3, 2)
    assert np.linalg.norm(r.sgs_state() - o.sgs_state()) / np.linalg.norm(o.sgs_state()) <= 1e-11
