"""Training the learned U-Net preconditioner on residual -> error pairs
harvested from plain (multigrid-preconditioned) CG solves of cut-cell urban
pressure problems, and using it in flexible CG.

    pairs = harvest_pairs(problems, cap=12)          # [(r_k, e_k)]
    net = train_unet(shape, pairs, steps=2000)
    mg.set_learned(net)                              # flexible CG with the network

    sim = urban_flow(n, seed, nboxes)                # the urban setup as a stepped flow
    net, losses, used = train_from_run(sim, steps=200, dt=0.2, cap=10)   # its own snapshots

A pair (r_k, e_k) is the residual after k CG iterations and the error
x* - x_k of that iterate against the converged solution, so A e_k = r_k.
"""
from __future__ import annotations

import numpy as np

from .cutcell import box_geometry, face_coefficients, pressure_rhs, random_boxes, urban_velocity
from .grids import regular_grid
from .spec import CoreSpec
from .multigrid import MGPreconditionedCG
from .unet import UNet, error_scale


def urban_geometry(n, seed, nboxes, delta=2.0):
    """The grid and cut-cell geometry of `nboxes` floor-standing boxes from
    `seed` on n cells of `delta` metres."""
    g = regular_grid(n, tuple(delta * v for v in n), halo=(3, 3, 3), bc_z="wall")
    return g, box_geometry(g, random_boxes(g, nboxes, seed=seed), nsub=4)


def urban_rhs(g, geom, noise_seed):
    """The right-hand side from a log-profile inflow with seeded noise."""
    u, v, w = urban_velocity(g, geom, seed=noise_seed)
    return pressure_rhs(geom, u, v, w)


def urban_problem(n, seed, nboxes, delta=2.0, noise_seed=None):
    """Face coefficients, right-hand side and fluid mask of the cut-cell
    urban pressure problem (noise from `noise_seed`, default `seed`)."""
    g, geom = urban_geometry(n, seed, nboxes, delta)
    fluid = (~geom.is_solid[g.interior]).astype(np.float32)
    return face_coefficients(geom), urban_rhs(g, geom, seed if noise_seed is None else noise_seed), fluid


def harvest_pairs(n, seeds, rhs_per_geometry, nboxes, cap=12, delta=2.0, tol=1e-8):
    """Residual -> error pairs (with the fluid mask of their geometry) from
    plain MG-preconditioned CG solves: for each geometry seed,
    `rhs_per_geometry` right-hand sides with fresh noise seeds."""
    out = []
    for s in seeds:
        g, geom = urban_geometry(n, s, nboxes, delta)
        fluid = (~geom.is_solid[g.interior]).astype(np.float32)
        mg = MGPreconditionedCG(n, (delta,) * 3, coeffs=face_coefficients(geom), tol=tol)
        for q in range(rhs_per_geometry):
            b = urban_rhs(g, geom, 1000 * s + q)
            x, st, pairs = mg.solve_harvest(b, cap)
            out.extend((r, e, fluid) for r, e in pairs if np.linalg.norm(r) > 0)
    return out


def train_unet(n, pairs, steps, lr=1e-3, seed=0, net=None, lr_final=1e-4):
    """Adam on the pairs (cycled in a seeded random order), the learning rate
    decaying geometrically from lr to lr_final.  Returns (net, losses)."""
    if net is None:
        net = UNet(n, seed=seed)
    net.set_out_scale(error_scale([(r, e) for r, e, _ in pairs]))
    rng = np.random.default_rng(seed)
    order = rng.permutation(len(pairs))
    losses = []
    mask_id = None
    for it in range(steps):
        r, e, fluid = pairs[order[it % len(pairs)]]
        if mask_id is not id(fluid):
            net.set_mask(fluid)
            mask_id = id(fluid)
        a = lr * (lr_final / lr) ** (it / max(steps - 1, 1))
        losses.append(net.train_step(r, e, a))
    return net, np.array(losses)


def train_streaming(n, seeds, rhs_per_geometry, nboxes, pairs_total, cap=12, lr=1e-3, lr_final=1e-4, seed=0,
                    delta=2.0, warm_pairs=None):
    """Harvest and train geometry by geometry (the pairs of one geometry in
    memory at a time): each harvested pair is used for one Adam step, up to
    `pairs_total` steps.  The output scale comes from the first geometry's
    pairs (or `warm_pairs`).  Returns (net, losses, pairs used)."""
    net = UNet(n, seed=seed)
    losses, used = [], 0
    rng = np.random.default_rng(seed)
    for gi, s in enumerate(seeds):
        g, geom = urban_geometry(n, s, nboxes, delta)
        fluid = (~geom.is_solid[g.interior]).astype(np.float32)
        mg = MGPreconditionedCG(n, (delta,) * 3, coeffs=face_coefficients(geom), tol=1e-8)
        pairs = []
        for q in range(rhs_per_geometry):
            _, _, ps = mg.solve_harvest(urban_rhs(g, geom, 1000 * s + q), cap)
            pairs.extend(p for p in ps if np.linalg.norm(p[0]) > 0)
        if gi == 0:
            net.set_out_scale(error_scale(warm_pairs or pairs))
        net.set_mask(fluid)
        for k in rng.permutation(len(pairs)):
            if used >= pairs_total:
                break
            a = lr * (lr_final / lr) ** (used / max(pairs_total - 1, 1))
            losses.append(net.train_step(pairs[k][0], pairs[k][1], a))
            used += 1
        del pairs, mg
        if used >= pairs_total:
            break
    return net, np.array(losses), used


def transfer(net, n, fluid):
    """The trained weights and output scale on a network for another grid
    (the convolutions are size-independent), with that grid's fluid mask."""
    other = UNet(n)
    other.set_params(net.params())
    other.set_mask(fluid)
    other.set_out_scale(net.out_scale)
    return other


def urban_flow(n, seed, nboxes, delta=2.0, precision="fp64", noise_seed=None, device=0):
    """The cut-cell urban setup as a stepped flow: the Boussinesq core on n
    cells of `delta` metres (periodic in x and y, walls in z), WENO-JS5 with
    Smagorinsky C_s = 0.17, no buoyancy, every projection the plain
    MG-preconditioned CG on the boxes' fractional face apertures to 1e-8;
    started from the log-profile inflow (5 m/s at 10 m, z0 = 0.1 m) with
    +-0.5 m/s noise from `noise_seed` (default `seed`), projected.  Returns
    (simulation, grid, geometry)."""
    from .simulation import Simulation
    g, geom = urban_geometry(n, seed, nboxes, delta)
    spec = CoreSpec(grid=g, advection="weno_js5", c_s=0.17, nu=0.0, solver="pcg", precision=precision)
    sim = Simulation(spec, device=device)
    sim.set_pcg(face_coefficients(geom, power=1), tol=1e-8, maxit=500)
    u, v, w = urban_velocity(g, geom, seed=seed if noise_seed is None else noise_seed)
    sim.set_state(u, v, w, g.zeros())
    sim.project()
    return sim, g, geom


def train_from_run(sim, steps, dt, cap=10, lr=1e-3, lr_final=1e-4, seed=0, net=None, fluid=None):
    """Train on the run's own snapshots: `steps` projected RK3 steps of `sim`
    (a PCG-projected simulation with the plain preconditioner), after each
    step the right-hand side of its last projection solved again by the plain
    MG-preconditioned CG with its first `cap` residual -> error pairs
    recorded (Simulation.pcg_harvest), each pair used at once for one Adam
    step (the rate decaying geometrically from lr to lr_final over the
    expected steps * cap pairs).  The output scale comes from the first
    step's pairs.  Returns (net, losses, pairs used)."""
    g = sim.grid
    n = (g.nx, g.ny, g.nz)
    if net is None:
        net = UNet(n, seed=seed)
    if fluid is not None:
        net.set_mask(np.asarray(fluid, dtype=np.float32))
    rng = np.random.default_rng(seed)
    total = max(steps * cap - 1, 1)
    losses, used = [], 0
    for it in range(steps):
        sim.step_rk3(dt, 1)
        _, _, pairs = sim.pcg_harvest(cap)
        pairs = [p for p in pairs if np.linalg.norm(p[0]) > 0]
        if it == 0:
            net.set_out_scale(error_scale(pairs))
        for k in rng.permutation(len(pairs)):
            a = lr * (lr_final / lr) ** (min(used, total) / total)
            losses.append(net.train_step(pairs[k][0], pairs[k][1], a))
            used += 1
    return net, np.array(losses), used
