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


def test_pairs_from_the_run_satisfy_the_operator():
    # the run's own snapshots: the right-hand side of the step's last
    # projection, solved again by the plain MG-preconditioned CG
    from aeolus_b200.cutcell import face_coefficients
    from aeolus_b200.learned import urban_flow
    sim, g, geom = urban_flow(N, seed=31, nboxes=3)
    sim.step_rk3(0.2, 2)
    b, x, pairs = sim.pcg_harvest(cap=8)
    st = sim.pcg_stats()
    assert st["status"] == "converged" and 2 <= len(pairs) <= 8
    o = OracleMGPCG(N, (H,) * 3, coeffs=face_coefficients(geom))
    rb = b - b.mean()
    assert np.linalg.norm(rb) > 0
    assert np.allclose(pairs[0][0], rb, rtol=0, atol=1e-14 * np.abs(b).max())
    assert np.linalg.norm(rb - o.apply(x)) <= 1.02e-8 * np.linalg.norm(rb)
    for r, e in pairs:
        assert np.linalg.norm(o.apply(e) - r) <= 1e-7 * np.linalg.norm(rb)
    # the step goes on after a harvest, and pairs come from plain solves only
    sim.step_rk3(0.2, 1)
    assert sim.pcg_stats()["status"] == "converged"
    from aeolus_b200.unet import UNet
    net = UNet(N)
    net.set_mask((~geom.is_solid[g.interior]).astype(np.float32))
    sim.set_learned(net, 0.9)
    with pytest.raises(RuntimeError):
        sim.pcg_harvest(cap=4)
    sim.set_learned(None)
    sim.close()


def test_network_trained_on_the_run_cuts_iterations():
    # trained on 160 pairs of a 20-step spin-up of one geometry, then used
    # on the projections of a run over a geometry of a fresh seed
    from aeolus_b200.learned import train_from_run, transfer, urban_flow
    sim, g, geom = urban_flow(N, seed=41, nboxes=3)
    net, losses, used = train_from_run(sim, steps=20, dt=0.2, cap=8,
                                       fluid=(~geom.is_solid[g.interior]).astype(np.float32))
    sim.close()
    assert used >= 100 and losses[-30:].mean() < 0.6 * losses[:30].mean()
    its = {}
    for name in ("identity", "learned"):
        t, tg, tgeom = urban_flow(N, seed=777, nboxes=3)
        fluid = (~tgeom.is_solid[tg.interior]).astype(np.float32)
        t.step_rk3(0.2, 1)
        b, _, _ = t.pcg_harvest(cap=1)
        from aeolus_b200.cutcell import face_coefficients
        from aeolus_b200.multigrid import MGPreconditionedCG
        s = MGPreconditionedCG(N, (H,) * 3, coeffs=face_coefficients(tgeom), tol=1e-8, maxit=2000,
                               precond="identity" if name == "identity" else "vcycle")
        if name == "learned":
            s.set_learned(transfer(net, N, fluid), stagnation=0.98)
        x, st = s.solve(b)
        assert st["status"] == "converged", st
        its[name] = st["iterations"]
        t.close()
    assert its["learned"] < 0.5 * its["identity"], its
