"""The multigrid / MG-preconditioned CG oracle against the reference's own
test cases (test/multigrid.jl:9-100, test/support/multigrid_cases.jl) and a
dense solve; the cut-cell geometry of axis-aligned boxes against exact
fractions.  CPU only."""
import numpy as np
import pytest

from oracle.mgpcg import OracleMGPCG

from aeolus_b200 import regular_grid
from aeolus_b200.cutcell import box_geometry, face_coefficients, cutcell_divergence, pressure_rhs


def cutcell_coeffs(nx, ny, nz, block=((4, 10), (8, 14), (0, 6))):
    """test/support/multigrid_cases.jl:12-27 (0-based, half-open block):
    every face of the solid block closed, plus partly open faces."""
    cx, cy, cz = np.ones((nz, ny, nx + 1)), np.ones((nz, ny + 1, nx)), np.ones((nz + 1, ny, nx))
    (i0, i1), (j0, j1), (k0, k1) = block
    cx[k0:k1, j0:j1, i0:i1 + 1] = 0
    cy[k0:k1, j0:j1 + 1, i0:i1] = 0
    cz[k0:k1 + 1, j0:j1, i0:i1] = 0
    cx[0:7, :, 3] *= 0.3
    cy[0:7, 7, :] *= 0.6
    cz[7, :, :] *= 0.8
    return cx, cy, cz


def cutcell_source(b, block=((4, 10), (8, 14), (0, 6))):
    """test/support/multigrid_cases.jl:31-36: zero in the solid, zero mean
    over the fluid."""
    (i0, i1), (j0, j1), (k0, k1) = block
    solid = np.zeros(b.shape, dtype=bool)
    solid[k0:k1, j0:j1, i0:i1] = True
    b[solid] = 0
    b[~solid] -= b[~solid].sum() / np.count_nonzero(~solid)
    return b


def grid_fn(n, f, h=None):
    nx, ny, nz = n
    h = h or (1.0 / nx, 1.0 / ny, 1.0 / nz)
    z, y, x = np.meshgrid((np.arange(nz) + 0.5) * h[2], (np.arange(ny) + 0.5) * h[1], (np.arange(nx) + 0.5) * h[0],
                          indexing="ij")
    return f(x, y, z)


def test_manufactured_periodic_solution_and_level_count():
    n = (16, 16, 16)
    phi = grid_fn(n, lambda x, y, z: np.sin(2 * np.pi * x) * np.cos(2 * np.pi * y) * np.sin(2 * np.pi * z))
    s = OracleMGPCG(n, (1 / 16,) * 3, bc=("periodic",) * 3, tol=1e-12, maxit=60)
    src = s.apply(phi)
    out, st = s.mg_solve(src)
    assert st["status"] == "converged"
    assert np.abs(out - phi).max() < 1e-9
    assert s.nlevels >= 3


def test_cycle_count_is_grid_independent_and_geometric():
    res = []
    for N in (16, 32):
        rng = np.random.default_rng(1234)
        rhs = rng.standard_normal((N, N, N))
        rhs -= rhs.mean()
        s = OracleMGPCG((N,) * 3, (1 / N,) * 3, tol=1e-8, maxit=60)
        # history: run cycle by cycle
        hist = []
        for c in range(1, 7):
            s.p.maxit = c
            s.p.tol = 0.0
            s2 = OracleMGPCG((N,) * 3, (1 / N,) * 3, tol=0.0, maxit=c)
            hist.append(s2.mg_solve(rhs)[1]["residual"])
        _, st = s.mg_solve(rhs)
        res.append((st["iterations"] if st["status"] == "converged" else 10 ** 9,
                    max(hist[i + 1] / hist[i] for i in range(5))))
    assert res[1][0] <= res[0][0] + 3
    assert res[1][1] < 0.5


def test_variable_coefficient_manufactured_solution():
    N = 8
    h = 1.0 / N
    c = lambda z: 1.0 + 2.0 * z
    zc = (np.arange(N) + 0.5) * h
    zf = np.arange(N + 1) * h
    cx = np.broadcast_to(c(zc)[:, None, None], (N, N, N + 1)).copy()
    cy = np.broadcast_to(c(zc)[:, None, None], (N, N + 1, N)).copy()
    cz = np.broadcast_to(c(zf)[:, None, None], (N + 1, N, N)).copy()
    s = OracleMGPCG((N,) * 3, (h,) * 3, coeffs=(cx, cy, cz), tol=1e-10, maxit=80)
    phi = grid_fn((N,) * 3, lambda x, y, z: np.sin(2 * np.pi * x) * np.cos(2 * np.pi * y) * np.cos(np.pi * z))
    phi -= phi.mean()
    rhs = s.apply(phi)
    rhs -= rhs.mean()
    out, st = s.mg_solve(rhs)
    assert st["status"] == "converged"
    assert np.abs(out - out.mean() - phi).max() < 1e-7


def test_mgcg_convergence_is_independent_of_the_rhs_scale():
    i, j, k = np.meshgrid(np.arange(1, 9), np.arange(1, 9), np.arange(1, 9), indexing="ij")
    b0 = (np.sin(0.7 * i) * np.cos(1.3 * j) + 0.1 * np.sin(0.9 * k) * i / 8).transpose(2, 1, 0)
    sols = []
    for scale in (1.0, 1e-6):
        s = OracleMGPCG((8, 8, 8), (250 / 8, 250 / 8, 100 / 8), tol=1e-10)
        x, st = s.solve(scale * b0)
        sols.append(x / scale)
    assert np.allclose(sols[1], sols[0], rtol=1e-8, atol=1e-8 * np.abs(sols[0]).max())


def test_zero_rhs():
    s = OracleMGPCG((16, 16, 16), (1.0,) * 3, tol=1e-11, maxit=60)
    x, st = s.mg_solve(np.zeros((16, 16, 16)))
    assert st["status"] == "zero_rhs" and not x.any()
    x, st = s.solve(np.zeros((16, 16, 16)))
    assert st["status"] == "zero_rhs" and st["iterations"] == 0 and not x.any()


@pytest.mark.parametrize("precond", ["vcycle", "identity"])
def test_cutcell_mgcg_matches_a_dense_solve(precond):
    n = (16, 16, 8)
    cx, cy, cz = cutcell_coeffs(*n, block=((4, 10), (8, 14), (0, 4)))
    rng = np.random.default_rng(303)
    b = cutcell_source(rng.standard_normal(n[::-1]), block=((4, 10), (8, 14), (0, 4)))
    h = (1000 / 16, 1000 / 16, 200 / 8)
    s = OracleMGPCG(n, h, coeffs=(cx, cy, cz), tol=1e-12, maxit=400, precond=precond)
    x, st = s.solve(b)
    assert st["status"] == "converged"
    # dense operator from unit vectors; solve on the fluid cells
    N = b.size
    A = np.zeros((N, N))
    e = np.zeros(N)
    for q in range(N):
        e[q] = 1.0
        A[:, q] = s.apply(e.reshape(b.shape)).ravel()
        e[q] = 0.0
    assert np.allclose(A, A.T, atol=1e-12 * np.abs(A).max())
    fluid = np.abs(np.diag(A)) > 0
    xf = np.linalg.lstsq(A[np.ix_(fluid, fluid)], b.ravel()[fluid], rcond=None)[0]
    xs = x.ravel()[fluid]
    d = (xs - xs.mean()) - (xf - xf.mean())
    assert np.abs(d).max() <= 1e-8 * np.abs(xf).max()
    assert np.linalg.norm(A @ x.ravel() - b.ravel()) <= 1e-11 * np.linalg.norm(b)


def test_cutcell_reference_case_converges_with_mg_and_mgcg():
    n = (64, 64, 32)
    h = (1000 / 64, 1000 / 64, 200 / 32)
    cx, cy, cz = cutcell_coeffs(*n)
    rng = np.random.default_rng(303)
    b = cutcell_source(rng.standard_normal(n[::-1]))
    s = OracleMGPCG(n, h, coeffs=(cx, cy, cz), tol=1e-10)
    x, st = s.solve(b)
    assert st["status"] == "converged" and st["iterations"] < 40
    r = b - b.mean() - s.apply(x)
    assert np.linalg.norm(r) <= 1e-10 * np.linalg.norm(b - b.mean()) * 1.0001
    mg = OracleMGPCG(n, h, coeffs=(cx, cy, cz), tol=1e-10, maxit=200)
    xm, stm = mg.mg_solve(b)
    assert stm["status"] == "converged"
    fluid = np.ones(b.shape, dtype=bool)
    fluid[0:6, 8:14, 4:10] = False
    d = (x - xm)[fluid]
    assert np.abs(d - d.mean()).max() <= 1e-7 * np.abs(x[fluid]).max()


def test_coefficient_coarsening_is_the_four_face_mean():
    n = (8, 8, 8)
    rng = np.random.default_rng(5)
    cx, cy, cz = rng.random((8, 8, 9)), rng.random((8, 9, 8)), rng.random((9, 8, 8))
    s = OracleMGPCG(n, (1.0,) * 3, coeffs=(cx, cy, cz))
    assert s.nlevels == 2 and s.level_dims(1) == (4, 4, 4)
    Cx, Cy, Cz = s.level_coeff(1)
    # coarse x-face I sits on fine face 2I; its four fine faces tile it
    ref = 0.25 * (cx[0::2, 0::2, 0::2] + cx[0::2, 1::2, 0::2] + cx[1::2, 0::2, 0::2] + cx[1::2, 1::2, 0::2])
    assert np.allclose(Cx, ref, rtol=0, atol=1e-15)
    refz = 0.25 * (cz[0::2, 0::2, 0::2] + cz[0::2, 0::2, 1::2] + cz[0::2, 1::2, 0::2] + cz[0::2, 1::2, 1::2])
    assert np.allclose(Cz, refz, rtol=0, atol=1e-15)


# ---------------------------------------------------------------------------
# cut-cell geometry of boxes (src/CutCell.jl:243-319, :398-493)

def test_box_geometry_fractions_are_exact_for_a_sub_cell_aligned_box():
    g = regular_grid((16, 16, 8), (32.0, 32.0, 16.0), halo=(3, 3, 3), bc_z="wall")
    box = [(4.5, 11.0, 6.0, 9.5, 0.0, 5.5)]    # faces on the nsub = 4 sub-lattice (0.5 m)
    geom = box_geometry(g, box, nsub=4)
    hx, hy, hz = g.halo
    I = (slice(hz, hz + 8), slice(hy, hy + 16), slice(hx, hx + 16))
    vol = geom.vol_frac[I]
    # the exact overlap volume of each cell with the box, plus the ground
    xc = np.arange(16) * 2.0
    def ov(a0, a1, lo, hi):
        return np.clip(np.minimum(a1, hi) - np.maximum(a0, lo), 0, None) / (a1 - a0)
    fx, fy = ov(xc, xc + 2, 4.5, 11.0), ov(xc, xc + 2, 6.0, 9.5)
    fz = ov(np.arange(8) * 2.0, np.arange(8) * 2.0 + 2, 0.0, 5.5)
    exact = 1.0 - fz[:, None, None] * fy[None, :, None] * fx[None, None, :]
    exact[exact <= 0] = 0
    assert np.allclose(vol, exact, atol=1e-15)
    # the floor face is closed (ground), lateral faces open above the box
    az = geom.az[hz, hy:hy + 16, hx:hx + 16]
    assert not az.any()
    assert geom.ax[hz + 7, hy + 3, hx + 3] == 1.0


def test_geometry_consistency_and_compatible_rhs():
    g = regular_grid((32, 32, 16), (64.0, 64.0, 32.0), halo=(3, 3, 3), bc_z="wall")
    boxes = [(10.0, 22.3, 5.0, 17.9, 0.0, 13.7), (30.0, 41.0, 30.0, 50.0, 0.0, 21.0),
             (58.0, 70.0, 20.0, 30.0, 0.0, 9.0)]           # the last wraps across x
    geom = box_geometry(g, boxes, nsub=4)
    solid = geom.is_solid
    # every face touching a solid cell is closed
    assert not (geom.ax[:, :, 1:][solid[:, :, 1:] | solid[:, :, :-1]]).any()
    assert not (geom.az[1:][solid[1:] | solid[:-1]]).any()
    assert (geom.vol_eff[~solid] >= geom.vol_min).all() and not geom.vol_eff[solid].any()
    # periodic images: the wrapped box appears on both sides
    hx, hy, hz = g.halo
    assert geom.vol_frac[hz + 1, hy + 12, hx + 1] == 0 and geom.vol_frac[hz + 1, hy + 12, hx + 30] == 0
    cx, cy, cz = face_coefficients(geom)
    assert np.array_equal(cx[:, :, 0], cx[:, :, -1]) and np.array_equal(cy[:, 0, :], cy[:, -1, :])
    rng = np.random.default_rng(2)
    u, v, w = (rng.standard_normal(g.storage_shape) for _ in range(3))
    b = pressure_rhs(geom, u, v, w)
    assert abs(b.sum()) < 1e-10 * np.abs(b).sum()
    assert not b[solid[hz:hz + 16, hy:hy + 32, hx:hx + 32]].any()
