"""The GPU multigrid-preconditioned CG (include/aeolus_b200_mgpcg.h) against
the oracle's restatement of MGPreconditionedCG / mg_solve! / pcg!
(src/Multigrid.jl, src/Backends.jl:1511-1589), on the reference's own
multigrid test cases (test/multigrid.jl, test/support/multigrid_cases.jl)
and on a cut-cell urban geometry.

Tolerances: the operator is the same FP64 arithmetic (1e-14); one V-cycle
agrees to rounding (1e-11, both deflated to zero mean); a converged FP64
solve takes the same iteration count (within one, the test sits on a
threshold) and agrees to 1e-9; the FP32-mixed solve reaches the same
||r|| <= tol ||b|| measured in FP64 and agrees with FP64 to 1e-6.
"""
import numpy as np
import pytest

from oracle.mgpcg import OracleMGPCG
from test_mgpcg_oracle import cutcell_coeffs, cutcell_source, grid_fn

from aeolus_b200 import regular_grid
from aeolus_b200.cutcell import box_geometry, face_coefficients, pressure_rhs, random_boxes, urban_velocity

pytestmark = pytest.mark.gpu


def MG(*a, **k):
    from aeolus_b200.multigrid import MGPreconditionedCG
    return MGPreconditionedCG(*a, **k)


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


REF_N = (64, 64, 32)
REF_H = (1000 / 64, 1000 / 64, 200 / 32)


def ref_case():
    cx, cy, cz = cutcell_coeffs(*REF_N)
    rng = np.random.default_rng(303)
    b = cutcell_source(rng.standard_normal(REF_N[::-1]))
    return (cx, cy, cz), b


def test_operator_matches_the_oracle():
    rng = np.random.default_rng(1)
    (cx, cy, cz), _ = ref_case()
    x = rng.standard_normal(REF_N[::-1])
    for coeffs, bc in ((None, ("periodic", "periodic", "neumann")), ((cx, cy, cz), ("neumann", "neumann", "neumann")),
                       ((cx, cy, cz), ("periodic",) * 3)):
        g, o = MG(REF_N, REF_H, coeffs=coeffs, bc=bc), OracleMGPCG(REF_N, REF_H, coeffs=coeffs, bc=bc)
        assert rel(g.apply(x), o.apply(x)) < 1e-14


def test_hierarchy_matches_the_oracle():
    g, o = MG((256, 256, 96), (2.0,) * 3), OracleMGPCG((256, 256, 96), (2.0,) * 3)
    assert g.nlevels == o.nlevels == 5
    assert g.level_dims() == [o.level_dims(l) for l in range(o.nlevels)]


@pytest.mark.parametrize("bc", [("periodic", "periodic", "neumann"), ("neumann", "neumann", "neumann"),
                                ("periodic", "periodic", "periodic")])
def test_one_vcycle_matches_the_oracle(bc):
    coeffs, b = ref_case()
    g, o = MG(REF_N, REF_H, coeffs=coeffs, bc=bc), OracleMGPCG(REF_N, REF_H, coeffs=coeffs, bc=bc)
    zg, zo = g.precondition(b), o.precondition(b)
    assert rel(zg, zo) < 1e-11


@pytest.mark.parametrize("n,bc,precision", [
    ((40, 24, 10), ("periodic",) * 3, "fp64"),          # coarsest 20 x 12 x 5: an odd periodic axis
    ((64, 64, 12), ("periodic", "periodic", "neumann"), "fp64"),   # coarsest 32 x 32 x 6 outside shared memory
    ((64, 64, 12), ("periodic", "periodic", "neumann"), "fp32_mixed"),
])
def test_coarsest_level_variants_match_the_oracle(n, bc, precision):
    rng = np.random.default_rng(8)
    nx, ny, nz = n
    cx, cy, cz = (0.2 + rng.random(s) for s in ((nz, ny, nx + 1), (nz, ny + 1, nx), (nz + 1, ny, nx)))
    cx[..., -1] = cx[..., 0]
    cy[:, -1, :] = cy[:, 0, :]
    if bc[2] == "periodic":
        cz[-1] = cz[0]
    b = rng.standard_normal((nz, ny, nx))
    g = MG(n, (1.0, 1.0, 1.0), coeffs=(cx, cy, cz), bc=bc, precision=precision)
    o = OracleMGPCG(n, (1.0, 1.0, 1.0), coeffs=(cx, cy, cz), bc=bc)
    assert g.level_dims() == [o.level_dims(l) for l in range(o.nlevels)]
    zg, zo = g.precondition(b), o.precondition(b)
    assert rel(zg, zo) < (1e-11 if precision == "fp64" else 1e-5)


@pytest.mark.parametrize("coded,bc,nu,precision", [
    (True, ("periodic", "periodic", "neumann"), (2, 2), "fp64"),
    (True, ("periodic", "periodic", "neumann"), (2, 2), "fp32_mixed"),
    (True, ("neumann", "neumann", "neumann"), (3, 1), "fp64"),
    (False, ("periodic", "periodic", "neumann"), (2, 2), "fp64"),
])
def test_large_level_vcycle_matches_the_oracle(coded, bc, nu, precision):
    """One V-cycle at 128 x 128 x 48 in each coefficient form of the smoother
    (one-byte codes on the finest level, per-face values below it, or the
    constant Laplacian), periodic or mirrored sides, and odd sweep counts."""
    n = (128, 128, 48)
    coeffs, b = urban_problem(n, seed=5, nboxes=10) if coded else (None, np.random.default_rng(6).standard_normal(n[::-1]))
    g = MG(n, (2.0,) * 3, coeffs=coeffs, bc=bc, nu1=nu[0], nu2=nu[1], precision=precision)
    o = OracleMGPCG(n, (2.0,) * 3, coeffs=coeffs, bc=bc, nu1=nu[0], nu2=nu[1])
    zg, zo = g.precondition(b), o.precondition(b)
    assert rel(zg, zo) < (1e-11 if precision == "fp64" else 1e-5)


def test_cutcell_mgcg_solve_matches_the_oracle():
    coeffs, b = ref_case()
    g = MG(REF_N, REF_H, coeffs=coeffs, tol=1e-10)
    o = OracleMGPCG(REF_N, REF_H, coeffs=coeffs, tol=1e-10)
    xg, sg = g.solve(b)
    xo, so = o.solve(b)
    assert sg["status"] == so["status"] == "converged"
    assert abs(sg["iterations"] - so["iterations"]) <= 1
    assert abs(sg["bnorm"] - so["bnorm"]) <= 1e-13 * so["bnorm"]
    assert rel(xg, xo) < 1e-9
    assert abs(xg.mean()) < 1e-12 * np.abs(xg).max()


def test_plain_cg_matches_the_oracle():
    n, h = (32, 32, 16), (1.0, 1.0, 1.0)
    cx, cy, cz = cutcell_coeffs(*n, block=((4, 10), (8, 14), (0, 6)))
    rng = np.random.default_rng(4)
    b = cutcell_source(rng.standard_normal(n[::-1]), block=((4, 10), (8, 14), (0, 6)))
    g = MG(n, h, coeffs=(cx, cy, cz), tol=1e-10, maxit=500, precond="identity")
    o = OracleMGPCG(n, h, coeffs=(cx, cy, cz), tol=1e-10, maxit=500, precond="identity")
    xg, sg = g.solve(b)
    xo, so = o.solve(b)
    assert sg["status"] == so["status"] == "converged"
    assert abs(sg["iterations"] - so["iterations"]) <= 2
    assert rel(xg, xo) < 1e-8


def jacobi_inverse(n, h, coeffs, bc):
    """1 / diag of the fine operator: -sum of c / h^2 over the faces, a Neumann
    boundary face contributing nothing; 0 on a cell with every face closed."""
    nx, ny, nz = n
    cx, cy, cz = coeffs
    d = np.zeros((nz, ny, nx))
    for c, ax, hh, b in ((cx, 2, h[0], bc[0]), (cy, 1, h[1], bc[1]), (cz, 0, h[2], bc[2])):
        lo = np.take(c, range(0, c.shape[ax] - 1), axis=ax).copy()
        hi = np.take(c, range(1, c.shape[ax]), axis=ax).copy()
        if b == "neumann":
            np.moveaxis(lo, ax, 0)[0] = 0
            np.moveaxis(hi, ax, 0)[-1] = 0
        d += (lo + hi) / hh ** 2
    return np.where(d > 0, -1.0 / np.where(d > 0, d, 1.0), 0.0)


def test_jacobi_pcg_solves_to_the_tolerance_and_sits_between_cg_and_mgpcg():
    """The Jacobi-preconditioned CG of the density-weighted projection
    (DensityWeightedPoissonSolver, src/components/urban/pressure_solver.jl:18-20):
    z = r / diag(A) exactly, the solve reaches ||r|| <= tol ||b|| (measured with
    the oracle's operator), agrees with the MG-preconditioned solution and
    takes fewer iterations than plain CG, more than MG-PCG. The two solutions
    are compared on the open cells, each less its mean there."""
    coeffs, b = ref_case()
    bc = ("periodic", "periodic", "neumann")
    invd = jacobi_inverse(REF_N, REF_H, coeffs, bc)
    g = MG(REF_N, REF_H, coeffs=coeffs, tol=1e-10, maxit=2000, precond="jacobi")
    z = g.precondition(b)
    zr = b * invd
    assert rel(z, zr - zr.mean()) < 1e-14
    o = OracleMGPCG(REF_N, REF_H, coeffs=coeffs, tol=1e-10)
    xj, sj = g.solve(b)
    assert sj["status"] == "converged"
    r = b - b.mean() - o.apply(xj)
    assert np.linalg.norm(r) <= 1.01e-10 * np.linalg.norm(b - b.mean())
    xm, sm = MG(REF_N, REF_H, coeffs=coeffs, tol=1e-10).solve(b)
    _, si = MG(REF_N, REF_H, coeffs=coeffs, tol=1e-10, maxit=2000, precond="identity").solve(b)
    fl = invd != 0      # a cell with every face closed is in the null space: its value is arbitrary
    assert rel(xj[fl] - xj[fl].mean(), xm[fl] - xm[fl].mean()) < 1e-7
    assert sm["iterations"] < sj["iterations"] < si["iterations"]
    xf, sf = MG(REF_N, REF_H, coeffs=coeffs, tol=1e-8, maxit=2000, precond="jacobi",
                precision="fp32_mixed").solve(b)
    assert sf["status"] == "converged"
    r = b - b.mean() - o.apply(xf)
    assert np.linalg.norm(r) <= 1.01e-8 * np.linalg.norm(b - b.mean())


def test_mg_cycles_match_the_oracle_and_the_manufactured_solution():
    n = (16, 16, 16)
    phi = grid_fn(n, lambda x, y, z: np.sin(2 * np.pi * x) * np.cos(2 * np.pi * y) * np.sin(2 * np.pi * z))
    o = OracleMGPCG(n, (1 / 16,) * 3, bc=("periodic",) * 3, tol=1e-12, maxit=60)
    g = MG(n, (1 / 16,) * 3, bc=("periodic",) * 3, tol=1e-12, maxit=60)
    src = o.apply(phi)
    xg, sg = g.mg_solve(src)
    xo, so = o.mg_solve(src)
    assert sg["status"] == "converged" and abs(sg["iterations"] - so["iterations"]) <= 1
    assert np.abs(xg - phi).max() < 1e-9
    coeffs, b = ref_case()
    g = MG(REF_N, REF_H, coeffs=coeffs, tol=1e-10, maxit=200)
    o = OracleMGPCG(REF_N, REF_H, coeffs=coeffs, tol=1e-10, maxit=200)
    xg, sg = g.mg_solve(b)
    xo, so = o.mg_solve(b)
    assert sg["status"] == so["status"] == "converged"
    assert abs(sg["iterations"] - so["iterations"]) <= 1
    assert rel(xg, xo) < 1e-8


def test_zero_rhs_and_rhs_scale():
    g = MG((16, 16, 16), (1.0,) * 3, tol=1e-11, maxit=60)
    x, st = g.solve(np.zeros((16, 16, 16)))
    assert st["status"] == "zero_rhs" and st["iterations"] == 0 and not x.any()
    x, st = g.mg_solve(np.zeros((16, 16, 16)))
    assert st["status"] == "zero_rhs" and not x.any()
    i, j, k = np.meshgrid(np.arange(1, 9), np.arange(1, 9), np.arange(1, 9), indexing="ij")
    b0 = (np.sin(0.7 * i) * np.cos(1.3 * j) + 0.1 * np.sin(0.9 * k) * i / 8).transpose(2, 1, 0)
    sols = []
    for scale in (1.0, 1e-6):
        s = MG((8, 8, 8), (250 / 8, 250 / 8, 100 / 8), tol=1e-10)
        x, st = s.solve(scale * b0)
        sols.append(x / scale)
    assert np.allclose(sols[1], sols[0], rtol=1e-8, atol=1e-8 * np.abs(sols[0]).max())


def urban_problem(n, seed, nboxes):
    g = regular_grid(n, (2.0 * n[0], 2.0 * n[1], 2.0 * n[2]), halo=(3, 3, 3), bc_z="wall")
    geom = box_geometry(g, random_boxes(g, nboxes, seed=seed), nsub=4)
    u, v, w = urban_velocity(g, geom, seed=seed)
    return face_coefficients(geom), pressure_rhs(geom, u, v, w)


@pytest.mark.parametrize("precision", ["fp64", "fp32_mixed"])
def test_urban_cutcell_solve_to_1e8(precision):
    n = (128, 128, 48)
    coeffs, b = urban_problem(n, seed=11, nboxes=10)
    o = OracleMGPCG(n, (2.0,) * 3, coeffs=coeffs, tol=1e-8)
    g = MG(n, (2.0,) * 3, coeffs=coeffs, tol=1e-8, precision=precision)
    xg, sg = g.solve(b)
    xo, so = o.solve(b)
    assert sg["status"] == "converged" and so["status"] == "converged"
    r = b - b.mean() - o.apply(xg)
    assert np.linalg.norm(r) <= 1.01e-8 * np.linalg.norm(b - b.mean())
    if precision == "fp64":
        assert abs(sg["iterations"] - so["iterations"]) <= 1
        assert rel(xg, xo) < 1e-8
    else:
        assert sg["iterations"] <= so["iterations"] + 2
        assert rel(xg, xo) < 1e-6


def test_device_pointer_solve_equals_the_host_solve():
    import torch
    coeffs, b = ref_case()
    g = MG(REF_N, REF_H, coeffs=coeffs, tol=1e-10)
    xh, sh = g.solve(b)
    bd = torch.from_numpy(b).cuda()
    xd = torch.empty_like(bd)
    sd = g.solve_device(bd.data_ptr(), xd.data_ptr())
    assert sd["iterations"] == sh["iterations"]
    assert np.array_equal(xd.cpu().numpy(), xh)


def test_rejects_unsupported_configurations():
    with pytest.raises(ValueError):
        MG((16, 16, 16), (1.0,) * 3, bc=("periodic", "dirichlet", "neumann"))
    with pytest.raises(ValueError):
        MG((250, 250, 125), (1.0,) * 3)        # coarsest 125 x 125 x 125 is above one block's level
