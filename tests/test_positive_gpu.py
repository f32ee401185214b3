"""The CUDA positivity-preserving advection (aeo_advect_positive) against the
oracle's restatement of advect_positive! (src/AdvectionSchemes.jl:1100-1160).

FP64: relative L2 <= 1e-11 of the oracle's tendency (sharp fields, the
limiter active), WENO-Z5 and WENO-JS5, periodic z and walls; the forward-Euler
update non-negative; the device entry point equals the host one.  FP32-mixed
(the arithmetic in FP32): within 1e-5 of the oracle and non-negative to FP32
rounding.
"""
import numpy as np
import pytest

from oracle.oracle import OracleSimulation
from positive_cases import case, grid, spec

pytestmark = pytest.mark.gpu


def Sim(sp):
    from aeolus_b200.simulation import Simulation
    return Simulation(sp)


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("scheme", ["weno_z5", "weno_js5"])
@pytest.mark.parametrize("bc_z", ["periodic", "wall"])
def test_fp64_matches_the_oracle(scheme, bc_z):
    g = grid(bc_z=bc_z)
    u, v, w, phi, dt = case(g, 11)
    base = np.random.default_rng(2).standard_normal(g.storage_shape)
    o = OracleSimulation(spec(g)).advect_positive(u, v, w, phi, dt, scheme=scheme, tend=base)
    s = Sim(spec(g))
    t = s.advect_positive(u, v, w, phi, dt, scheme=scheme, tend=base)
    assert rel(t[g.interior], o[g.interior]) < 1e-11
    t0 = s.advect_positive(u, v, w, phi, dt, scheme=scheme, accumulate=False)[g.interior]
    assert (phi[g.interior] + dt * t0).min() >= -1e-14


def test_fp32_mixed_close_to_the_oracle():
    g = grid(n=(64, 32, 16))
    u, v, w, phi, dt = case(g, 12)
    o = OracleSimulation(spec(g)).advect_positive(u, v, w, phi, dt, accumulate=False)[g.interior]
    t = Sim(spec(g, "fp32_mixed")).advect_positive(u, v, w, phi, dt, accumulate=False)[g.interior]
    assert rel(t, o) < 1e-5
    assert (phi[g.interior] + dt * t).min() >= -1e-6


def test_device_entry_point_equals_the_host_one():
    import torch
    g = grid()
    u, v, w, phi, dt = case(g, 13)
    s = Sim(spec(g))
    host = s.advect_positive(u, v, w, phi, dt, accumulate=False)
    dev = [torch.from_numpy(a).cuda() for a in (u, v, w, phi)]
    tend = torch.zeros(g.storage_shape, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    s.advect_positive_device(*dev, tend, dt, accumulate=False)
    s.synchronize()
    assert np.array_equal(tend.cpu().numpy()[g.interior], host[g.interior])
