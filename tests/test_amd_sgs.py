"""The anisotropic minimum-dissipation closure (AMDClosure /
compute_amd_coefficients!, src/operators/sgs_amd_vreman.jl:18-90, :109-212,
:325-354): nu_t from the scaled-gradient production with the buoyancy term
weighted by min(1, 1/Ri), theta's own kappa_t from the scalar production, the
nu_t / Pr_t fallback where the theta gradient vanishes, the constant C = c_s.

Oracle (CPU): nu_t and kappa_t equal a numpy statement of _amd_point on a
random stratified field; nu_t is exactly zero in a pure shear flow u(z) (the
closure's laminar-flow property) where Smagorinsky's is not; kappa_t is
unchanged by theta -> a theta + b; on the sound-proof core the buoyancy
parameter is g/theta_bar(z_k) of each level.  GPU (`-m gpu`): steps with the
AMD closure match the oracle to 1e-11 (FP64; theta compared as its departure
from theta0), on both cores, and FP32-mixed to 1e-5; the adaptive dt with the
eddy coefficients binding matches the oracle's pick to 1e-12.
"""
import numpy as np
import pytest

from aeolus_b200 import CoreSpec, regular_grid
from oracle.oracle import OracleSimulation

FIELDS = ("u", "v", "w", "theta")
C_AMD = 0.3
TH0 = 300.0


def grid():
    return regular_grid((16, 16, 16), (1.0, 1.0, 0.5), halo=(3, 3, 3), bc_z="wall")


def spec(g, sgs="amd", advection="centred", precision="fp64", c_s=C_AMD, theta0=TH0):
    return CoreSpec(grid=g, c_s=c_s, sgs=sgs, theta0=theta0, advection=advection, precision=precision)


def state(g, seed=4, amp=1.0):
    """Random velocities and a stably stratified theta with noise (walls in z)."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = g.size
    th = np.full(g.storage_shape, TH0)
    z = g.znodes("c")
    th[g.interior] += 2.0 * z[:, None, None] + 0.1 * rng.standard_normal((nz, ny, nx))
    u, v, w = g.zeros(), g.zeros(), g.zeros()
    u[g.interior] = amp * rng.standard_normal((nz, ny, nx))
    v[g.interior] = amp * rng.standard_normal((nz, ny, nx))
    w[g.interior] = amp * rng.standard_normal((nz, ny, nx))
    w[g.halo[2]] = 0.0
    return u, v, w, th


def amd_numpy(g, u, v, w, th, C, pr_t, bg):
    """_velocity_gradient_at, _scalar_gradient_at and _amd_point on the
    interior (storage arrays with filled halos): (nu_t, kappa_t)."""
    hx, hy, hz = g.halo
    nx, ny, nz = g.size

    def sh(a, di, dj, dk):
        return a[hz + dk:hz + dk + nz, hy + dj:hy + dj + ny, hx + di:hx + di + nx]
    idx, idy, idz = 1 / g.dx, 1 / g.dy, 1 / g.dz
    G = np.empty((3, 3, nz, ny, nx))
    G[0, 0] = (sh(u, 1, 0, 0) - sh(u, 0, 0, 0)) * idx
    G[1, 1] = (sh(v, 0, 1, 0) - sh(v, 0, 0, 0)) * idy
    G[2, 2] = (sh(w, 0, 0, 1) - sh(w, 0, 0, 0)) * idz
    G[0, 1] = ((sh(u, 0, 1, 0) + sh(u, 1, 1, 0)) - (sh(u, 0, -1, 0) + sh(u, 1, -1, 0))) * (0.25 * idy)
    G[1, 0] = ((sh(v, 1, 0, 0) + sh(v, 1, 1, 0)) - (sh(v, -1, 0, 0) + sh(v, -1, 1, 0))) * (0.25 * idx)
    G[0, 2] = ((sh(u, 0, 0, 1) + sh(u, 1, 0, 1)) - (sh(u, 0, 0, -1) + sh(u, 1, 0, -1))) * (0.25 * idz)
    G[2, 0] = ((sh(w, 1, 0, 0) + sh(w, 1, 0, 1)) - (sh(w, -1, 0, 0) + sh(w, -1, 0, 1))) * (0.25 * idx)
    G[1, 2] = ((sh(v, 0, 0, 1) + sh(v, 0, 1, 1)) - (sh(v, 0, 0, -1) + sh(v, 0, 1, -1))) * (0.25 * idz)
    G[2, 1] = ((sh(w, 0, 1, 0) + sh(w, 0, 1, 1)) - (sh(w, 0, -1, 0) + sh(w, 0, -1, 1))) * (0.25 * idy)
    gt = np.stack([(sh(th, 1, 0, 0) - sh(th, -1, 0, 0)) * (0.5 * idx),
                   (sh(th, 0, 1, 0) - sh(th, 0, -1, 0)) * (0.5 * idy),
                   (sh(th, 0, 0, 1) - sh(th, 0, 0, -1)) * (0.5 * idz)])
    d2 = np.array([g.dx ** 2, g.dy ** 2, g.dz ** 2])[:, None, None, None]

    def sdot(a, b):
        return (d2 * a * b).sum(axis=0)
    S = 0.5 * (G + G.transpose(1, 0, 2, 3, 4))
    P = sum(sdot(G[i], G[j]) * S[i, j] for i in range(3) for j in range(3))
    B = bg * sdot(G[2], gt)
    D = (G ** 2).sum(axis=(0, 1))
    kd = (gt ** 2).sum(axis=0)
    N2 = abs(bg) * np.sqrt(kd)
    Bw = np.where(D >= N2, B, B * (D / np.where(N2 > 0, N2, 1.0)))
    Q = sum(sdot(G[i], gt) * gt[i] for i in range(3))
    nu = np.where(D > 0, C * np.maximum(0.0, -P + Bw) / np.where(D > 0, D, 1.0), 0.0)
    ka = np.where(kd > 0, C * np.maximum(0.0, -Q) / np.where(kd > 0, kd, 1.0), nu / pr_t)
    return nu, ka


def test_oracle_coefficients_are_the_amd_point():
    g = grid()
    sp = spec(g)
    o = OracleSimulation(sp)
    o.set_state(*state(g))
    o.tendencies()
    nut, kt = o.get_field("nut")[g.interior], o.get_field("kt")[g.interior]
    f = [o.get_field(n) for n in FIELDS]
    nu, ka = amd_numpy(g, *f, C_AMD, sp.pr_t, sp.g / TH0)
    assert np.count_nonzero(nu) > nu.size // 4 and np.count_nonzero(ka) > ka.size // 4
    assert np.abs(nut - nu).max() <= 1e-12 * np.abs(nu).max()
    assert np.abs(kt - ka).max() <= 1e-12 * np.abs(ka).max()


def test_amd_vanishes_in_pure_shear():
    g = grid()
    z = g.znodes("c")
    u = g.zeros()
    u[g.interior] = np.sin(3 * z)[:, None, None]
    zero = g.zeros()
    th = np.full(g.storage_shape, TH0)
    for sgs, c_s, expect_zero in (("amd", C_AMD, True), ("smagorinsky", 0.17, False)):
        o = OracleSimulation(spec(g, sgs, c_s=c_s))
        o.set_state(u, zero, zero, th)
        o.tendencies()
        nut = o.get_field("nut")[g.interior]
        assert (np.abs(nut).max() == 0.0) == expect_zero, sgs


def test_kappa_is_invariant_under_an_affine_theta():
    """kappa_t is homogeneous of degree 0 in theta (no buoyancy: theta0 = 0)."""
    g = grid()
    u, v, w, th = state(g, seed=9)
    out = []
    for a, b in ((1.0, 0.0), (-2.5, 40.0)):
        o = OracleSimulation(spec(g, theta0=0.0))
        o.set_state(u, v, w, a * th + b)
        o.tendencies()
        out.append((o.get_field("nut")[g.interior], o.get_field("kt")[g.interior]))
    (n0, k0), (n1, k1) = out
    assert np.array_equal(n0, n1)
    assert np.abs(k1 - k0).max() <= 1e-12 * np.abs(k0).max()


def anelastic_spec(g, advection="centred", precision="fp64"):
    """The sound-proof core on the uniform wall-bounded grid: an exponential
    density and a stable theta_bar profile; the AMD buoyancy parameter is
    g/theta_bar(z_k) of the cell centres (sgs_buoyancy_parameter,
    src/operators/sgs_amd_vreman.jl:331-345)."""
    from aeolus_b200.reference_state import anelastic_profiles, exponential_density
    thc = 250.0 + 200.0 * g.znodes("c")
    prof = anelastic_profiles(g, exponential_density(g), thc)
    return CoreSpec(grid=g, core="anelastic", c_s=C_AMD, sgs="amd", advection=advection, precision=precision,
                    wc=prof["wc"], wf=prof["wf"], thf=prof["thf"], thc=thc)


def test_amd_needs_a_uniform_grid_and_centre_theta_on_the_sound_proof_core():
    from aeolus_b200 import stretched_grid, tanh_faces
    g = stretched_grid((16, 16, 16), (1.0, 1.0, 0.5), tanh_faces(16, 0.5, 1.5), halo=(3, 3, 3))
    with pytest.raises(ValueError):
        CoreSpec(grid=g, c_s=C_AMD, sgs="amd")
    n = 16
    with pytest.raises(ValueError):
        CoreSpec(grid=grid(), core="anelastic", c_s=C_AMD, sgs="amd", wc=np.ones(n + 6), wf=np.ones(n + 7))
    assert anelastic_spec(grid()).thc.shape == (n,)


def test_oracle_amd_on_the_sound_proof_core_uses_the_level_buoyancy():
    """nu_t and kappa_t of the sound-proof core are the AMD point with the
    buoyancy parameter of each level, g/theta_bar(z_k)."""
    g = grid()
    sp = anelastic_spec(g)
    o = OracleSimulation(sp)
    o.set_state(*state(g))
    o.tendencies()
    nut, kt = o.get_field("nut")[g.interior], o.get_field("kt")[g.interior]
    f = [o.get_field(n) for n in FIELDS]
    nu, ka = amd_numpy(g, *f, C_AMD, sp.pr_t, (sp.g / sp.thc)[:, None, None])
    assert np.abs(nut - nu).max() <= 1e-12 * np.abs(nu).max()
    assert np.abs(kt - ka).max() <= 1e-12 * np.abs(ka).max()
    nu0, _ = amd_numpy(g, *f, C_AMD, sp.pr_t, sp.g / TH0)
    assert np.abs(nu - nu0).max() > 1e-7 * np.abs(nu).max()   # the level values matter


@pytest.mark.gpu
@pytest.mark.parametrize("advection", ["centred", "weno_js5"])
def test_gpu_amd_steps_match_the_oracle(advection):
    from aeolus_b200.simulation import Simulation
    g = grid()
    st = state(g)
    sims = [OracleSimulation(spec(g, advection=advection)), Simulation(spec(g, advection=advection)),
            Simulation(spec(g, advection=advection, precision="fp32_mixed"))]
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
    sp = spec(g)
    nut = sims[1].get_field("nut")[g.interior]
    nu, _ = amd_numpy(g, *(sims[1].get_field(n) for n in FIELDS), C_AMD, sp.pr_t, sp.g / TH0)
    assert np.abs(nut - nu).max() <= 1e-12 * np.abs(nu).max()


@pytest.mark.gpu
def test_gpu_amd_on_the_sound_proof_core_matches_the_oracle():
    """theta starts on the reference profile plus a stable 2 K/m and noise;
    compared as its departure from theta_bar(z).  FP32 stores theta -
    theta_bar(bottom face): a stored range of ~100 K against a ~1 K
    departure, so theta's FP32 bar is 1e-4 (the velocities' 1e-5)."""
    from aeolus_b200.simulation import Simulation
    g = grid()
    u, v, w, th = state(g)
    sp = anelastic_spec(g)
    thb = np.broadcast_to(sp.thc[:, None, None], (g.nz, g.ny, g.nx))
    th = th.copy()
    th[g.interior] += thb - TH0
    sims = [OracleSimulation(sp), Simulation(anelastic_spec(g)), Simulation(anelastic_spec(g, precision="fp32_mixed"))]
    out = []
    for s in sims:
        s.set_state(u, v, w, th)
        s.project()   # the flux form's theta tendency depends on theta's storage offset unless div(W u) = 0
        s.step_rk3(2e-3, 3)
        f = {n: s.get_field(n)[g.interior] for n in FIELDS}
        f["theta"] = f["theta"] - thb
        out.append(f)
    ora, g64, g32 = out
    e64 = {n: np.linalg.norm(g64[n] - ora[n]) / np.linalg.norm(ora[n]) for n in FIELDS}
    assert all(e <= 1e-11 for e in e64.values()), e64
    e32 = {n: np.linalg.norm(g32[n] - g64[n]) / np.linalg.norm(g64[n]) for n in FIELDS}
    assert all(e <= (1e-4 if n == "theta" else 1e-5) for n, e in e32.items()), e32
    sp = anelastic_spec(g)
    nut = sims[1].get_field("nut")[g.interior]
    nu, _ = amd_numpy(g, *(sims[1].get_field(n) for n in FIELDS), C_AMD, sp.pr_t, (sp.g / sp.thc)[:, None, None])
    assert np.abs(nut - nu).max() <= 1e-12 * np.abs(nu).max()


@pytest.mark.gpu
def test_gpu_amd_adaptive_dt_matches_the_oracle():
    """A strong closure constant makes the eddy coefficients bind the pick
    (nu + nu_t for the diffusive limit, max(nu_t, kappa_t) with the closure's
    own kappa_t for the SGS limit)."""
    from aeolus_b200._lib import LIMITERS
    from aeolus_b200.simulation import CFLConstraints, Simulation
    g = grid()
    sp = spec(g, c_s=30.0)
    s, o = Simulation(sp), OracleSimulation(sp)
    for x in (s, o):
        x.set_state(*state(g, amp=0.05))
    c = CFLConstraints(C_advective=0.5)
    d = s.cfl_diagnostics(c)
    dto, lim = o.adaptive_dt(c)
    assert d["limiter"] == LIMITERS[lim] and d["limiter"] in ("diffusive", "sgs")
    assert abs(d["dt"] - dto) <= 1e-12 * dto
