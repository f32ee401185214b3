"""The reference's decaying-turbulence DNS fixture as a known answer for the
step (`test/fixtures/dns_decay.jl:8-30`, checked by
`validation/apriori_sgs.jl:128-141`): centred advection, molecular viscosity
nu = 0.018 (48/N)^(4/3), the projected SSP-RK3 at CFL 0.5.  The reference
records, per grid: the dissipation peak at t ~ 0.99 / 1.45 / 1.85 at
32^3 / 48^3 / 64^3, the derivative skewness in -0.6 ... -0.35 once the
cascade is under way (reached within t ~ 0.4), the one-step energy budget
dK/dt = -eps to within 2 % (1.7e-4 measured), a monotone decay and
k_max eta >= 1.5 at 48^3 (1.54).  The oracle's step must reproduce these
numbers (it restates the reference's operators; a mis-weighted viscous or
advective term moves the budget, the peak or the skewness), and the FP64
CUDA step must reproduce the oracle's history."""
import numpy as np
import pytest

import dns_decay_case as dns
from aeolus_b200 import CoreSpec

PEAK = {32: 0.99, 48: 1.45, 64: 1.85}


def check_fixture(h, n):
    i = int(np.argmax(h["eps"]))
    assert 0 < i < len(h["eps"]) - 1, "the dissipation peak must lie inside the run"
    assert abs(h["t"][i] - PEAK[n]) < 0.15, (n, h["t"][i])
    late = h["t"] >= 0.4
    assert np.all((h["S"][late] >= -0.6) & (h["S"][late] <= -0.35)), (h["S"][late].min(), h["S"][late].max())
    assert np.abs(h["budget_err"]).max() <= 0.02
    assert np.all(np.diff(h["K"]) < 0)
    if n >= 48:
        assert dns.kmax_eta(h, n, dns.dns_nu(n)) >= 1.5


def oracle_history(n, t_end):
    from oracle.oracle import OracleSimulation
    g, st = dns.dns_grid_and_state(n)
    nu = dns.dns_nu(n)
    o = OracleSimulation(CoreSpec(grid=g, advection="centred", nu=nu))
    o.set_state(*st)
    h = dns.run(o, g, nu, t_end=t_end)
    o.close()
    return h


@pytest.mark.parametrize("n,t_end", [(32, 1.6), (48, 2.0)])
def test_oracle_reproduces_the_dns_fixture(n, t_end):
    check_fixture(oracle_history(n, t_end), n)


def test_random_field_is_solenoidal_with_the_shell_energies():
    """`isotropic_random_field!`: zero discrete divergence, K = sum E(k_n) dk
    before the rescale to K = 3/2 (src/operators/spectra.jl:84-113)."""
    n = 24
    E = lambda k: k ** 4 * np.exp(-2 * (k / 1.5) ** 2)
    u, v, w = dns.random_field(n, E, seed=3)
    h = 2 * np.pi / n
    div = (np.roll(u, -1, 2) - u + np.roll(v, -1, 1) - v + np.roll(w, -1, 0) - w) / h
    assert np.abs(div).max() < 1e-12 * np.abs(u).max() / h
    K = 0.5 * float(np.mean(u * u) + np.mean(v * v) + np.mean(w * w))
    assert abs(K - sum(E(q) for q in range(1, n // 2 + 1))) < 1e-12 * K


@pytest.mark.gpu
@pytest.mark.parametrize("n,t_end", [(32, 1.6), (64, 2.4)])
def test_cuda_step_reproduces_the_dns_fixture(n, t_end):
    """The CUDA transforms take powers of two, so the fixture runs at the
    reference's 32^3 and 64^3 (its 48^3 on the oracle only)."""
    from aeolus_b200.simulation import Simulation
    g, st = dns.dns_grid_and_state(n)
    nu = dns.dns_nu(n)
    s = Simulation(CoreSpec(grid=g, advection="centred", nu=nu))
    s.set_state(*st)
    h = dns.run(s, g, nu, t_end=t_end)
    s.close()
    check_fixture(h, n)
    if n == 32:   # the whole history equals the oracle's (same dt sequence)
        ho = oracle_history(n, t_end)
        assert len(ho["t"]) == len(h["t"])
        for k in ("K", "eps", "S"):
            assert np.abs(h[k] - ho[k]).max() <= 1e-9 * np.abs(ho[k]).max(), k
