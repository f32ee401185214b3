"""Flexible CG preconditioned by the learned U-Net on cut-cell urban
pressure problems: trained on the GPU on residual -> error pairs of plain
MG-preconditioned CG solves (training geometries), tested on a geometry of
a fresh seed.  Every solve must reach the same ||r|| <= 1e-8 ||b||; the
network must cut the iteration count of the CG it preconditions (against
CG with no preconditioner, the method without it); an untrained network
that stagnates hands over to the multigrid cycle and the solve still
converges to the same answer."""
import numpy as np
import pytest

from oracle.mgpcg import OracleMGPCG

pytestmark = pytest.mark.gpu

N = (64, 64, 24)
H = 2.0


def test_learned_preconditioner_cuts_iterations_and_keeps_the_answer():
    from aeolus_b200.learned import harvest_pairs, train_unet, urban_problem, transfer
    from aeolus_b200.multigrid import MGPreconditionedCG
    pairs = harvest_pairs(N, seeds=(21, 22, 23, 24), rhs_per_geometry=4, nboxes=3, cap=12)
    assert len(pairs) >= 100
    net, losses = train_unet(N, pairs, steps=600, lr=1e-3, seed=0)
    assert losses[-50:].mean() < 0.5 * losses[:50].mean()
    coeffs, b, fluid = urban_problem(N, seed=777, nboxes=3)        # fresh geometry
    o = OracleMGPCG(N, (H,) * 3, coeffs=coeffs, tol=1e-8)
    plain = MGPreconditionedCG(N, (H,) * 3, coeffs=coeffs, tol=1e-8, maxit=2000, precond="identity")
    xp, sp = plain.solve(b)
    learned = MGPreconditionedCG(N, (H,) * 3, coeffs=coeffs, tol=1e-8, maxit=2000)
    learned.set_learned(transfer(net, N, fluid), stagnation=0.98)
    xl, sl = learned.solve(b)
    assert sl["status"] == "converged" and sp["status"] == "converged"
    rb = b - b.mean()
    assert np.linalg.norm(rb - o.apply(xl)) <= 1.02e-8 * np.linalg.norm(rb)
    assert sl["iterations"] < 0.5 * sp["iterations"], (sl, sp)
    xm, sm = MGPreconditionedCG(N, (H,) * 3, coeffs=coeffs, tol=1e-8).solve(b)
    f = fluid > 0
    d = (xl - xm)[f]
    assert np.abs(d - d.mean()).max() <= 1e-5 * np.abs(xm[f]).max()


def test_untrained_network_falls_back_to_the_cycle():
    from aeolus_b200.learned import urban_problem
    from aeolus_b200.multigrid import MGPreconditionedCG
    from aeolus_b200.unet import UNet
    coeffs, b, fluid = urban_problem(N, seed=5, nboxes=3)
    net = UNet(N, seed=9)
    net.set_mask(fluid)
    net.set_out_scale(1.0)
    s = MGPreconditionedCG(N, (H,) * 3, coeffs=coeffs, tol=1e-8, maxit=500)
    s.set_learned(net, stagnation=0.9)
    x, st = s.solve(b)
    assert st["status"] == "converged" and st["fallback_at"] >= 0
    o = OracleMGPCG(N, (H,) * 3, coeffs=coeffs, tol=1e-8)
    rb = b - b.mean()
    assert np.linalg.norm(rb - o.apply(x)) <= 1.02e-8 * np.linalg.norm(rb)


def test_harvested_pairs_satisfy_the_operator():
    from aeolus_b200.learned import urban_problem
    from aeolus_b200.multigrid import MGPreconditionedCG
    coeffs, b, fluid = urban_problem(N, seed=3, nboxes=3)
    s = MGPreconditionedCG(N, (H,) * 3, coeffs=coeffs, tol=1e-10)
    x, st, pairs = s.solve_harvest(b, cap=8)
    assert len(pairs) == min(st["iterations"] + 1, 8)
    o = OracleMGPCG(N, (H,) * 3, coeffs=coeffs)
    b0 = np.linalg.norm(pairs[0][0])          # slot 0: b - mean b
    assert np.allclose(pairs[0][0], b - b.mean(), rtol=0, atol=1e-14 * np.abs(b).max())
    for r, e in pairs:
        # A e_k = r_k up to the accuracy of the converged solution
        assert np.linalg.norm(o.apply(e) - r) <= 1e-8 * b0
