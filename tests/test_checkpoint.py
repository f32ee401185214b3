"""The checkpoint state mirror (aeolus_b200.checkpoint; checkpoint!,
checkpoint_payload, write_checkpoint, src/io/checkpoint.jl:346-473).

Host logic on the CPU, with the oracle's domain standing in for the device
domain (the same get_field / set_field interface): a written checkpoint reads
back equal, the write leaves no temporary file, a restart from it continues
the run exactly (the restarted steps equal the uninterrupted ones bit for
bit), a checkpoint of another mesh or other parameters is refused, and the
buffers of an earlier payload are refilled in place.  GPU (`-m gpu`): the
same restart property on the device domain.
"""
import os

import numpy as np
import pytest

from aeolus_b200 import CoreSpec, regular_grid
from aeolus_b200.checkpoint import (FIELDS, checkpoint, checkpoint_payload, read_checkpoint, restore,
                                    write_checkpoint)
from oracle.oracle import OracleSimulation


def spec(n=16, c_s=0.17, advection="weno_js5", sgs="smagorinsky", **kw):
    g = regular_grid((n, n, n), (1.0, 1.0, 0.5), halo=(3, 3, 3), bc_z="wall")
    return CoreSpec(grid=g, c_s=c_s, theta0=300.0, advection=advection, nu=1e-4, sgs=sgs, **kw)


def state(g, seed=3):
    rng = np.random.default_rng(seed)
    nx, ny, nz = g.size
    th = np.full(g.storage_shape, 300.0)
    th[g.interior] += 0.1 * rng.standard_normal((nz, ny, nx))
    u, v, w = g.zeros(), g.zeros(), g.zeros()
    for a in (u, v, w):
        a[g.interior] = 0.5 * rng.standard_normal((nz, ny, nx))
    w[g.halo[2]] = 0.0
    return u, v, w, th


def restart_matches(make, tmp_path, sp=None):
    sp = sp or spec()
    a = make(sp)
    a.set_state(*state(sp.grid))
    a.project()
    a.step_rk3(2e-3, 2)
    path = checkpoint(a, os.path.join(tmp_path, "run.ckpt"), t=4e-3, stepper={"dt_prev": 2e-3},
                      extra={"step": 2})
    assert not os.path.exists(path + ".tmp")
    a.step_rk3(2e-3, 2)
    b = make(sp)
    t, stepper = restore(b, path)
    assert t == 4e-3 and stepper == {"dt_prev": 2e-3}
    b.step_rk3(2e-3, 2)
    for n in ("u", "v", "w", "theta"):
        assert np.array_equal(a.get_field(n), b.get_field(n)), n
    if sp.sgs == "lagrangian":
        for x, y in zip(a.sgs_state(), b.sgs_state()):
            assert np.array_equal(x, y)
    if sp.sgs == "tke":
        assert np.array_equal(a.sgs_state(), b.sgs_state())


def test_written_checkpoint_reads_back(tmp_path):
    sp = spec()
    o = OracleSimulation(sp)
    o.set_state(*state(sp.grid))
    o.project()
    p = checkpoint_payload(o, t=1.5, extra={"note": "x"})
    path = write_checkpoint(os.path.join(tmp_path, "sub", "a.ckpt"), p)
    q = read_checkpoint(path)
    assert set(q["fields"]) == set(FIELDS)
    for n in FIELDS:
        assert np.array_equal(q["fields"][n], p["fields"][n])
    for k in ("format", "version", "mesh", "t", "parameters", "closure_type", "extra", "sim_type"):
        assert q[k] == p[k], k
    assert q["closure_type"] == "smagorinsky" and q["mesh"]["size"] == [16, 16, 16]


def test_restart_continues_the_run_exactly(tmp_path):
    restart_matches(OracleSimulation, str(tmp_path))


def test_restart_with_the_lagrangian_memories(tmp_path):
    """the closure's state (checkpoint_state = sgs_state) travels with the
    fields: the restarted run continues the memories bit for bit"""
    restart_matches(OracleSimulation, tmp_path, spec(c_s=0.5, sgs="lagrangian"))
    a = OracleSimulation(spec(c_s=0.5, sgs="lagrangian"))
    a.set_state(*state(a.grid))
    p = checkpoint(a, os.path.join(tmp_path, "lag.ckpt"))
    with pytest.raises(ValueError):
        restore(OracleSimulation(spec()), p, check_parameters=False)


def test_restart_with_the_tke(tmp_path):
    restart_matches(OracleSimulation, tmp_path, spec(c_s=0.1, sgs="tke", tke_e0=0.01))


def test_checkpoint_of_another_domain_is_refused(tmp_path):
    sp = spec()
    o = OracleSimulation(sp)
    o.set_state(*state(sp.grid))
    path = checkpoint(o, os.path.join(tmp_path, "a.ckpt"))
    with pytest.raises(ValueError, match="mesh"):
        restore(OracleSimulation(spec(n=8)), path)
    other = OracleSimulation(spec(c_s=0.1))
    with pytest.raises(ValueError, match="parameters"):
        restore(other, path)
    restore(other, path, check_parameters=False)
    bad = read_checkpoint(path)
    bad["format"] = "something else"
    with pytest.raises(ValueError):
        restore(o, bad)


def test_buffers_are_refilled_in_place():
    sp = spec()
    o = OracleSimulation(sp)
    o.set_state(*state(sp.grid))
    p1 = checkpoint_payload(o)
    o.step_rk3(2e-3, 1)
    p2 = checkpoint_payload(o, buffers=p1["fields"])
    for n in FIELDS:
        assert p2["fields"][n] is p1["fields"][n]
        assert np.array_equal(p2["fields"][n], o.get_field(n))


@pytest.mark.gpu
@pytest.mark.parametrize("sgs,c_s,kw", [("smagorinsky", 0.17, {}), ("lagrangian", 0.5, {}), ("tke", 0.1, {"tke_e0": 0.01})])
def test_gpu_restart_continues_the_run_exactly(tmp_path, sgs, c_s, kw):
    from aeolus_b200.simulation import Simulation
    restart_matches(Simulation, str(tmp_path), spec(c_s=c_s, sgs=sgs, **kw))
