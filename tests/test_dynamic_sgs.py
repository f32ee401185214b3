"""Dynamic Smagorinsky (DynamicSmagorinsky / compute_dynamic_smagorinsky_nut!,
src/Operators.jl:497-900, src/operators/sgs_closures.jl:425-462): the
Germano identity in Lilly's least-squares form with the 3 x 3 x 3 box test
filter (width ratio 3), plane-averaged per level and clipped to
[0, cs_max^2], cs_max passed as c_s; nu_t = C_s^2(z) Delta^2 |S| with
Delta^2 = (dx dy dz)^(2/3), kappa_t = nu_t / Pr_t.

Oracle (CPU): nu_t equals a numpy statement of the procedure on a random
field; with a small cs_max the clip binds and nu_t is the static
Smagorinsky nu_t of C_s = cs_max on every level the clip caps (and zero on
the levels of net backscatter).  GPU (`-m gpu`):
steps with the dynamic closure match the oracle to 1e-11 (FP64; walls and
periodic z; plane and local averaging) and FP32-mixed to 1e-5; the nu_t
diagnostic and the adaptive dt match the oracle.
"""
import numpy as np
import pytest

from aeolus_b200 import CoreSpec, regular_grid
from oracle.oracle import OracleSimulation

FIELDS = ("u", "v", "w", "theta")
CS_MAX = 0.5
TH0 = 300.0


def grid(bc_z="wall"):
    return regular_grid((16, 16, 16), (1.0, 1.0, 0.5), halo=(3, 3, 3), bc_z=bc_z)


def spec(g, sgs="dynamic", advection="centred", precision="fp64", c_s=CS_MAX, averaging="plane"):
    return CoreSpec(grid=g, c_s=c_s, sgs=sgs, theta0=TH0, advection=advection, precision=precision,
                    averaging=averaging)


def state(g, seed=5, amp=1.0):
    rng = np.random.default_rng(seed)
    nx, ny, nz = g.size
    th = np.full(g.storage_shape, TH0)
    th[g.interior] += 0.1 * rng.standard_normal((nz, ny, nx))
    u, v, w = g.zeros(), g.zeros(), g.zeros()
    # a smooth large-scale flow plus noise, so that the resolved stress has a
    # forward-scatter part on most levels
    z, y, x = np.meshgrid(g.znodes("c"), (np.arange(ny) + 0.5) / ny, (np.arange(nx) + 0.5) / nx, indexing="ij")
    u[g.interior] = amp * (np.sin(2 * np.pi * y) * np.cos(4 * np.pi * z) + 0.3 * rng.standard_normal((nz, ny, nx)))
    v[g.interior] = amp * (np.sin(2 * np.pi * x) + 0.3 * rng.standard_normal((nz, ny, nx)))
    w[g.interior] = amp * 0.3 * rng.standard_normal((nz, ny, nx))
    if g.bc_z == "wall":
        w[g.halo[2]] = 0.0
    return u, v, w, th


def dynamic_numpy(g, u, v, w, cs_max, local=False, parts=False):
    """_germano_pass1 / _germano_pass2 / _plane_cs2_body! (local:
    _local_cs2_body!) / _dynamic_nut_body! on storage arrays with filled
    halos: nu_t on the interior (parts: each cell's LM, MM, |S| and its
    cell-centred velocity instead)."""
    hx, hy, hz = g.halo
    nx, ny, nz = g.size

    def sh(a, di, dj, dk, s=1):      # interior + s shell cells
        return a[hz - s + dk:hz + nz + s + dk, hy - s + dj:hy + ny + s + dj, hx - s + di:hx + nx + s + di]
    idx, idy, idz = 1 / g.dx, 1 / g.dy, 1 / g.dz
    Uc = 0.5 * (sh(u, 0, 0, 0) + sh(u, 1, 0, 0))
    Vc = 0.5 * (sh(v, 0, 0, 0) + sh(v, 0, 1, 0))
    Wc = 0.5 * (sh(w, 0, 0, 0) + sh(w, 0, 0, 1))
    du_dx = (sh(u, 1, 0, 0) - sh(u, 0, 0, 0)) * idx
    dv_dy = (sh(v, 0, 1, 0) - sh(v, 0, 0, 0)) * idy
    dw_dz = (sh(w, 0, 0, 1) - sh(w, 0, 0, 0)) * idz
    du_dy = ((sh(u, 0, 1, 0) + sh(u, 1, 1, 0)) - (sh(u, 0, -1, 0) + sh(u, 1, -1, 0))) * (0.25 * idy)
    dv_dx = ((sh(v, 1, 0, 0) + sh(v, 1, 1, 0)) - (sh(v, -1, 0, 0) + sh(v, -1, 1, 0))) * (0.25 * idx)
    du_dz = ((sh(u, 0, 0, 1) + sh(u, 1, 0, 1)) - (sh(u, 0, 0, -1) + sh(u, 1, 0, -1))) * (0.25 * idz)
    dw_dx = ((sh(w, 1, 0, 0) + sh(w, 1, 0, 1)) - (sh(w, -1, 0, 0) + sh(w, -1, 0, 1))) * (0.25 * idx)
    dv_dz = ((sh(v, 0, 0, 1) + sh(v, 0, 1, 1)) - (sh(v, 0, 0, -1) + sh(v, 0, 1, -1))) * (0.25 * idz)
    dw_dy = ((sh(w, 0, 1, 0) + sh(w, 0, 1, 1)) - (sh(w, 0, -1, 0) + sh(w, 0, -1, 1))) * (0.25 * idy)
    S = [du_dx, dv_dy, dw_dz, 0.5 * (du_dy + dv_dx), 0.5 * (du_dz + dw_dx), 0.5 * (dv_dz + dw_dy)]
    ms = np.sqrt(2 * (S[0] ** 2 + S[1] ** 2 + S[2] ** 2) + 4 * (S[3] ** 2 + S[4] ** 2 + S[5] ** 2))
    q = [Uc, Vc, Wc, Uc * Uc, Vc * Vc, Wc * Wc, Uc * Vc, Uc * Wc, Vc * Wc] + S + [ms * s for s in S]

    def box(a):
        return sum(a[1 + c:1 + c + nz, 1 + b:1 + b + ny, 1 + d:1 + d + nx]
                   for c in (-1, 0, 1) for b in (-1, 0, 1) for d in (-1, 0, 1)) / 27
    t = [box(a) for a in q]
    Ut, Vt, Wt = t[0], t[1], t[2]
    L = [t[3] - Ut * Ut, t[4] - Vt * Vt, t[5] - Wt * Wt, t[6] - Ut * Vt, t[7] - Ut * Wt, t[8] - Vt * Wt]
    tr = (L[0] + L[1] + L[2]) / 3
    L[0], L[1], L[2] = L[0] - tr, L[1] - tr, L[2] - tr
    A = t[9:15]
    magSt = np.sqrt(2 * (A[0] ** 2 + A[1] ** 2 + A[2] ** 2) + 4 * (A[3] ** 2 + A[4] ** 2 + A[5] ** 2))
    d2 = (g.dx * g.dy * g.dz) ** (2 / 3)
    M = [2 * d2 * (t[15 + c] - 9.0 * magSt * A[c]) for c in range(6)]
    LM = L[0] * M[0] + L[1] * M[1] + L[2] * M[2] + 2 * (L[3] * M[3] + L[4] * M[4] + L[5] * M[5])
    MM = M[0] ** 2 + M[1] ** 2 + M[2] ** 2 + 2 * (M[3] ** 2 + M[4] ** 2 + M[5] ** 2)
    if parts:
        inner = (slice(1, -1),) * 3
        return LM, MM, ms[inner], (Uc[inner], Vc[inner], Wc[inner])
    if local:
        cs2 = np.where(MM > 0, np.clip(LM / np.where(MM > 0, MM, 1.0), 0.0, cs_max ** 2), 0.0)
        return cs2 * d2 * ms[1:-1, 1:-1, 1:-1], cs2
    lm, mm = LM.sum(axis=(1, 2)), MM.sum(axis=(1, 2))
    cs2 = np.where(mm > 0, np.clip(lm / np.where(mm > 0, mm, 1.0), 0.0, cs_max ** 2), 0.0)
    return cs2[:, None, None] * d2 * ms[1:-1, 1:-1, 1:-1], cs2


def test_oracle_nut_is_the_dynamic_procedure():
    g = grid()
    o = OracleSimulation(spec(g))
    o.set_state(*state(g))
    o.tendencies()
    nut = o.get_field("nut")[g.interior]
    ref, cs2 = dynamic_numpy(g, *(o.get_field(n) for n in ("u", "v", "w")), CS_MAX)
    assert np.count_nonzero(cs2) >= len(cs2) // 2 and cs2.max() < CS_MAX ** 2
    assert np.abs(nut - ref).max() <= 1e-12 * np.abs(ref).max()


def test_oracle_nut_with_local_averaging():
    """averaging = :local (src/Operators.jl:521-522, 873-880): every cell its
    own clipped L^d:M / M:M; noisy, so some cells clip at cs_max^2 and some at 0."""
    g = grid()
    o = OracleSimulation(spec(g, averaging="local"))
    o.set_state(*state(g))
    o.tendencies()
    nut = o.get_field("nut")[g.interior]
    ref, cs2 = dynamic_numpy(g, *(o.get_field(n) for n in ("u", "v", "w")), CS_MAX, local=True)
    assert np.count_nonzero(cs2 == 0) > 0 and np.count_nonzero((cs2 > 0) & (cs2 < CS_MAX ** 2)) > cs2.size // 4
    assert np.abs(nut - ref).max() <= 1e-12 * np.abs(ref).max()
    with pytest.raises(ValueError):
        spec(g, averaging="box")


def test_the_clip_gives_the_static_closure():
    g = grid()
    cs = 1e-3
    out = {}
    for sgs in ("dynamic", "smagorinsky"):
        o = OracleSimulation(spec(g, sgs, c_s=cs))
        o.set_state(*state(g))
        o.tendencies()
        out[sgs] = o.get_field("nut")[g.interior]
        vel = [o.get_field(n) for n in ("u", "v", "w")]    # halos filled
    _, cs2 = dynamic_numpy(g, *vel, cs)
    clipped = cs2 == cs ** 2
    assert clipped.sum() >= 3 and np.all(cs2[~clipped] == 0)   # forward scatter clipped, backscatter zeroed
    d, s = out["dynamic"], out["smagorinsky"]
    assert np.allclose(d[clipped], s[clipped], rtol=1e-12, atol=0)
    assert np.all(d[~clipped] == 0)


def test_dynamic_needs_a_uniform_grid_and_halos_of_two():
    from aeolus_b200 import stretched_grid, tanh_faces
    g = stretched_grid((16, 16, 16), (1.0, 1.0, 0.5), tanh_faces(16, 0.5, 1.5), halo=(3, 3, 3))
    with pytest.raises(ValueError):
        CoreSpec(grid=g, c_s=CS_MAX, sgs="dynamic")
    with pytest.raises(ValueError):
        CoreSpec(grid=regular_grid((16, 16, 16), (1.0,) * 3, halo=(1, 1, 1)), c_s=CS_MAX, sgs="dynamic")


@pytest.mark.gpu
@pytest.mark.parametrize("advection,bc_z,averaging", [("centred", "wall", "plane"), ("weno_js5", "wall", "plane"),
                                                      ("centred", "periodic", "plane"), ("centred", "wall", "local"),
                                                      ("weno_js5", "wall", "local"), ("centred", "periodic", "local")])
def test_gpu_dynamic_steps_match_the_oracle(advection, bc_z, averaging):
    from aeolus_b200.simulation import Simulation
    g = grid(bc_z)
    st = state(g)
    kw = dict(advection=advection, averaging=averaging)
    sims = [OracleSimulation(spec(g, **kw)), Simulation(spec(g, **kw)),
            Simulation(spec(g, precision="fp32_mixed", **kw))]
    out = []
    for s in sims:
        s.set_state(*st)
        s.project()
        s.step_rk3(2e-3, 3)
        f = {n: s.get_field(n)[g.interior] for n in FIELDS}
        f["theta"] = f["theta"] - TH0
        out.append(f)
    ora, g64, g32 = out
    e64 = {n: np.linalg.norm(g64[n] - ora[n]) / np.linalg.norm(ora[n]) for n in FIELDS}
    assert all(e <= 1e-11 for e in e64.values()), e64
    e32 = {n: np.linalg.norm(g32[n] - g64[n]) / np.linalg.norm(g64[n]) for n in FIELDS}
    assert all(e <= 1e-5 for e in e32.values()), e32
    nut = sims[1].get_field("nut")[g.interior]
    ref, _ = dynamic_numpy(g, *(sims[1].get_field(n) for n in ("u", "v", "w")), CS_MAX, local=averaging == "local")
    assert np.abs(nut - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.gpu
@pytest.mark.parametrize("averaging", ["plane", "local"])
def test_gpu_dynamic_adaptive_dt_matches_the_oracle(averaging):
    from aeolus_b200._lib import LIMITERS
    from aeolus_b200.simulation import CFLConstraints, Simulation
    g = grid()
    sp = spec(g, c_s=30.0, averaging=averaging)
    s, o = Simulation(sp), OracleSimulation(sp)
    for x in (s, o):
        x.set_state(*state(g, amp=0.05))
    c = CFLConstraints(C_advective=0.5)
    d = s.cfl_diagnostics(c)
    dto, lim = o.adaptive_dt(c)
    assert d["limiter"] == LIMITERS[lim]
    assert abs(d["dt"] - dto) <= 1e-12 * dto
