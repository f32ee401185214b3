"""Ghost-cell wall reconstruction, the wall shear stress and the wall laws.

CPU (host stencils + the oracle) restates the reference's checks
(test/cutcell.jl:14-176):
  * a cell cut in half by a plane: fractions 1/2, the apertures, the wetted
    area; the normal of a tilted plane;
  * the reconstruction of a field linear in the wall distance is exact
    (Dirichlet and Neumann), second order for a quadratic one (error ratio
    3.2 .. 4.8 under refinement), one ghost layer on a flat wall;
  * the resolved wall shear stress of u = alpha (z - z_w) is nu alpha;
  * small-cell merging conserves sum(vol_eff div) and gives the cluster one value;
and the wall laws (src/wall_models/laws.jl): Spalding's u+ = y+ in the
viscous sublayer and the log law far out, the rough log law, Monin-Obukhov
reducing to it when neutral.  `-m gpu`: the CUDA reconstruction (FP64 and
FP32 device fields, every location) and the stresses and slip velocities
of every law equal the oracle's on a sphere over a tilted plane.
"""
import math

import numpy as np
import pytest

from aeolus_b200 import regular_grid
from aeolus_b200.cutcell import cut_cell_geometry, cutcell_divergence
from aeolus_b200.ghost import MOSTWallLaw, RoughLogLaw, SpaldingLaw, build_ghost_stencils
from oracle import ghost as og


def zc(g, k):
    return (k - g.halo[2] + 0.5) * g.dz


def ghost_case(N, power, wall):
    g = regular_grid((4, 4, N), (1.0, 1.0, 1.0), halo=(2, 2, 2), bc_z="wall")
    zw = (N // 4 + 0.7) * g.dz
    geom = cut_cell_geometry(g, lambda x, y, z: z - zw)
    st = build_ghost_stencils(geom, "c")
    k = np.arange(g.storage_shape[0])
    f = np.broadcast_to((wall + (zc(g, k) - zw) ** power)[:, None, None], g.storage_shape).copy()
    f2 = og.reconstruct(f, st, wall_value=wall).ravel()
    exact = (wall + (zc(g, k) - zw) ** power)
    err = max(abs(f2[st.target[s]] - exact[st.k[s]]) for s in range(len(st)) if st.ghost[s])
    return err, int(st.ghost.sum()), g, zw, geom, st


def test_plane_cuts_a_cell_in_half():
    g = regular_grid((4, 4, 8), (1.0, 1.0, 1.0), halo=(2, 2, 2), bc_z="wall")
    zw = 0.5 + g.dz / 2
    geom = cut_cell_geometry(g, lambda x, y, z: z - zw)
    K, J, I = 2 + 4, slice(2, 6), slice(2, 6)
    assert np.allclose(geom.vol_frac[K, J, I], 0.5, atol=1e-12)
    assert np.allclose(geom.ax[K, J, I], 0.5, atol=1e-12)
    assert np.all(geom.az[K, J, I] == 0) and np.all(geom.az[K + 1, J, I] == 1)
    assert np.allclose(geom.area[K, J, I], g.dx * g.dy, atol=1e-14)
    gt = cut_cell_geometry(g, lambda x, y, z: z - 0.3 - 0.2 * x)
    inner = (slice(2, 10), slice(2, 6), slice(2, 6))
    cut = gt.is_cut[inner]
    assert cut.any()
    assert np.abs(gt.nx[inner][cut] + 0.2 / math.sqrt(1.04)).max() < 1e-12


def test_reconstruction_is_exact_for_linear_and_second_order():
    err, nghost, g, zw, geom, st = ghost_case(16, 1, 3.0)
    assert nghost == 16                                # one ghost layer, 4 x 4 columns
    assert err < 1e-12
    k = np.arange(g.storage_shape[0])
    f = np.broadcast_to((2.0 + 3.0 * (zc(g, k) - zw))[:, None, None], g.storage_shape).copy()
    f2 = og.reconstruct(f, st, wall_flux=1.5, kappa=0.5).ravel()
    exact = 2.0 + 3.0 * (zc(g, k) - zw)
    assert max(abs(f2[st.target[s]] - exact[st.k[s]]) for s in range(len(st))) < 1e-12
    e16, e32 = ghost_case(16, 2, 0.0)[0], ghost_case(32, 2, 0.0)[0]
    assert 3.2 < e16 / e32 < 4.8                       # second order


def test_resolved_wall_shear_stress_on_the_true_normal():
    err, nghost, g, zw, geom, st = ghost_case(16, 1, 0.0)
    nu, alpha = 1.5e-2, 2.5
    k = np.arange(g.storage_shape[0])
    u = np.broadcast_to((alpha * (zc(g, k) - zw))[:, None, None], g.storage_shape).copy()
    tau = og.wall_shear_stress(u, g.zeros(), g.zeros(), st, nu)
    assert np.allclose(tau, nu * alpha, rtol=1e-10)


def test_small_cell_merging_conserves_the_divergence():
    g = regular_grid((4, 4, 4), (1.0, 1.0, 1.0), halo=(2, 2, 2), bc_z="wall")
    geom = cut_cell_geometry(g, lambda x, y, z: z - 0.26, nsub=4)
    k, j, i = 2 + 1, 2 + 1, 2 + 1                     # turn this cell into a sliver
    geom.vol_frac[k, j, i] = 1e-4
    geom.vol_eff[k, j, i] = geom.vol_min
    geom.is_small[k, j, i] = True
    geom.is_cut[k, j, i] = True
    n3, n2, n1 = geom.vol_frac.shape
    geom.merge_target[k, j, i] = ((k + 1) * n2 + j) * n1 + i
    rng = np.random.default_rng(3)
    u, v, w = (rng.standard_normal(g.storage_shape) for _ in range(3))
    ve = geom.vol_eff[g.interior]
    d0 = cutcell_divergence(geom, u, v, w, redistribute=False)
    d1 = cutcell_divergence(geom, u, v, w, redistribute=True)
    assert abs((ve * d1).sum() - (ve * d0).sum()) <= 1e-12 * abs((ve * d0).sum()) + 1e-14
    assert d1[k - 2, j - 2, i - 2] == pytest.approx(d1[k - 1, j - 2, i - 2])


def test_small_cells_get_the_most_open_neighbour():
    g = regular_grid((4, 4, 4), (1.0, 1.0, 1.0), halo=(2, 2, 2), bc_z="wall")
    geom = cut_cell_geometry(g, lambda x, y, z: z - 0.48, nsub=8, vol_min=0.2)   # 1/8-full cells under the plane
    small = np.argwhere(geom.is_small)
    assert len(small) > 0
    n3, n2, n1 = geom.vol_frac.shape
    for k, j, i in small:
        t = geom.merge_target[k, j, i]
        if t < 0:
            continue
        kt, jt, it = t // (n1 * n2), (t // n1) % n2, t % n1
        assert abs(kt - k) + abs(jt - j) + abs(it - i) == 1
        assert geom.vol_frac[kt, jt, it] >= geom.vol_frac[k, j, i]


def test_wall_laws():
    sp = SpaldingLaw()
    nu, h = 1e-5, 1e-3
    U = 1e-4                                            # y+ << 1: the viscous sublayer, u_tau^2 = nu U / h
    ut = og.friction_velocity(sp, U, h, nu)
    assert ut ** 2 == pytest.approx(nu * U / h, rel=1e-3)
    U, h = 5.0, 10.0                                    # far out: the log law
    ut = og.friction_velocity(sp, U, h, nu)
    yp = h * ut / nu
    assert U / ut == pytest.approx(math.log(yp) / sp.kappa + sp.B, rel=1e-4)
    rl = RoughLogLaw(0.1)
    assert og.friction_velocity(rl, 5.0, 10.0) == pytest.approx(0.4 * 5.0 / math.log(100.0), rel=1e-15)
    assert og.friction_velocity(MOSTWallLaw(0.1), 5.0, 10.0) == pytest.approx(og.friction_velocity(rl, 5.0, 10.0),
                                                                               rel=1e-12)
    stable = og.friction_velocity(MOSTWallLaw(0.1, L=50.0), 5.0, 10.0)
    unstable = og.friction_velocity(MOSTWallLaw(0.1, L=-50.0), 5.0, 10.0)
    assert stable < og.friction_velocity(rl, 5.0, 10.0) < unstable


# ------------------------------------------------------------------ GPU ---
def sphere_over_plane(n=8):
    g = regular_grid((n, n, n), (1.0, 1.0, 1.0), halo=(2, 2, 2), bc_z="wall")
    geom = cut_cell_geometry(g, lambda x, y, z: np.minimum(
        z - 0.18 - 0.12 * x, np.sqrt((x - 0.5) ** 2 + (y - 0.45) ** 2 + (z - 0.6) ** 2) - 0.22))
    return g, geom


@pytest.mark.gpu
@pytest.mark.parametrize("loc", ["c", "fx", "fy", "fz"])
def test_gpu_reconstruction_matches_the_oracle(loc):
    import torch
    from aeolus_b200.ghost import DeviceGhost
    g, geom = sphere_over_plane()
    st = build_ghost_stencils(geom, loc)
    assert st.ghost.sum() > 10
    dg = DeviceGhost(st)
    f = np.random.default_rng(5).standard_normal(g.storage_shape)
    for kw in ({"wall_value": 0.7}, {"wall_flux": -1.3, "kappa": 0.4}):
        ref = og.reconstruct(f, st, **kw)
        got = dg.reconstruct(f, **kw)
        assert np.abs(got - ref).max() <= 1e-14 * np.abs(ref).max(), kw
        # in place on a device field, FP64 and FP32
        t = torch.from_numpy(f.copy()).cuda()
        dg.reconstruct_device(t.data_ptr(), **kw)
        torch.cuda.synchronize()
        assert np.abs(t.cpu().numpy() - ref).max() <= 1e-14 * np.abs(ref).max()
        t32 = torch.from_numpy(f.astype(np.float32)).cuda()
        dg.reconstruct_device(t32.data_ptr(), fp32=True, **kw)
        torch.cuda.synchronize()
        ref32 = og.reconstruct(f.astype(np.float32).astype(np.float64), st, **kw)
        assert np.abs(t32.cpu().numpy() - ref32).max() <= 1e-6 * np.abs(ref32).max()
    dg.close()


@pytest.mark.gpu
def test_gpu_wall_stress_and_slip_match_the_oracle():
    from aeolus_b200.ghost import DeviceGhost
    g, geom = sphere_over_plane()
    st = build_ghost_stencils(geom, "c", probe_factor=2.0)
    dg = DeviceGhost(st)
    rng = np.random.default_rng(9)
    u, v, w = (rng.standard_normal(g.storage_shape) for _ in range(3))
    nu = 1.5e-5
    tau, slip = dg.wall_stress(u, v, w, nu=nu)
    assert np.allclose(tau, og.wall_shear_stress(u, v, w, st, nu), rtol=1e-12, atol=1e-300)
    assert not slip.any()
    for law in (SpaldingLaw(), RoughLogLaw(1e-4), MOSTWallLaw(1e-4, L=30.0), MOSTWallLaw(1e-4, L=-30.0)):
        nue = nu + 1e-3
        tau, slip = dg.wall_stress(u, v, w, nu=nu, law=law, nu_eff=nue)
        rt, rs = og.wall_stress_and_slip(u, v, w, st, law, nu=nu, nu_eff=nue)
        assert np.allclose(tau, rt, rtol=1e-10, atol=0), type(law).__name__
        assert np.allclose(slip, rs, rtol=1e-9, atol=1e-12 * np.abs(rs).max()), type(law).__name__
    with pytest.raises(ValueError):
        dg.wall_stress(u, v, w, nu=nu, law=RoughLogLaw(10.0), nu_eff=nu)   # probes below z0
    dg.close()
