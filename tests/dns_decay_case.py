"""The reference's decaying-turbulence DNS fixture, restated for the tests.

`test/fixtures/dns_decay.jl:1-30, 120-206` (Aeolus.jl): a triply periodic
2 pi box at N^3, a random solenoidal field of spectrum E(k) ~ k^4
exp(-2 (k/1.5)^2) scaled to K = 3/2 (u' = 1), nu = 0.018 (48/N)^(4/3),
stepped by the projected SSP-RK3 with centred advection and no SGS model at
dt = 0.5 dx / max|u_i| (`dns_step!`, :153-164).  Per step it records the
mean kinetic energy K, the viscous sink of the discrete Laplacian
eps = -nu <u_i lap u_i> (`_dns_epsilon`, :52-63), the derivative skewness
from the staggered forward differences (`velocity_derivative_skewness`,
:71-97) and the one-step budget error -(dK/dt)/mean(eps) - 1.  The
reference records for 48^3: the dissipation peak at t ~ 1.45, the skewness
in -0.6 ... -0.35 once developed, |budget error| <= 0.02 per step
(`validation/apriori_sgs.jl:128-141`, 1.7e-4 measured at 96^3), a
monotone decay, k_max eta >= 1.5 over the run (1.54 at the peak).

The start restates `isotropic_random_field!` (src/operators/spectra.jl:115-183):
complex Gaussian vectors per mode projected normal to the discrete staggered
divergence, Hermitian symmetry, every shell rescaled to hold exactly
E(k_n) dk of face energy, the half-cell phase shift to the faces.  The
reference draws with Julia's Xoshiro, which cannot be reproduced here; the
draws come from numpy's generator, so the statistics, not the bits, are what
the fixture's numbers pin.
"""
import numpy as np

KP = 1.5
NU48 = 0.018


def random_field(n, spectrum, seed=1):
    """`isotropic_random_field!` on the triply periodic 2 pi box at n^3:
    interior arrays (u, v, w) [k][j][i] on their faces."""
    L = 2 * np.pi
    h = L / n
    dk = 2 * np.pi / L
    nmax = int(np.floor((np.pi / h) / dk + 1e-9))
    m = np.fft.fftfreq(n, 1.0 / n)
    kz, ky, kx = np.meshgrid(m * dk, m * dk, m * dk, indexing="ij")
    mz, my, mx = np.meshgrid(m, m, m, indexing="ij")
    nyq = (np.abs(mx) == n // 2) | (np.abs(my) == n // 2) | (np.abs(mz) == n // 2)
    shell = np.rint(np.sqrt(kx ** 2 + ky ** 2 + kz ** 2) / dk).astype(np.int64)
    shell[nyq | (shell > nmax)] = 0
    on = shell > 0
    rng = np.random.default_rng(seed)
    # randn(ComplexF64): real and imaginary parts each of variance 1/2
    r = [(rng.standard_normal(kx.shape) + 1j * rng.standard_normal(kx.shape)) / np.sqrt(2) for _ in range(3)]
    S = [np.sin(k * h / 2) / h for k in (kx, ky, kz)]
    den = np.where(on, S[0] ** 2 + S[1] ** 2 + S[2] ** 2, 1.0)
    alpha = (S[0] * r[0] + S[1] * r[1] + S[2] * r[2]) / den
    C = [np.where(on, r[j] - alpha * S[j], 0.0) for j in range(3)]
    # Hermitian symmetry: 0.5 (C(k) + conj C(-k))
    neg = (-np.arange(n)) % n
    C = [0.5 * (c + np.conj(c[np.ix_(neg, neg, neg)])) for c in C]
    norm = 0.5 / float(n ** 3) ** 2
    e = norm * (np.abs(C[0]) ** 2 + np.abs(C[1]) ** 2 + np.abs(C[2]) ** 2)
    have = np.bincount(shell.ravel(), weights=e.ravel(), minlength=nmax + 1)
    want = np.array([max(float(spectrum(q * dk)), 0.0) * dk for q in range(nmax + 1)])
    scale = np.where(have > 0, np.sqrt(want / np.where(have > 0, have, 1.0)), 0.0)
    scale[0] = 0.0
    out = []
    for j, k in enumerate((kx, ky, kz)):
        A = C[j] * scale[shell] * np.exp(-1j * k * h / 2)
        out.append(np.real(np.fft.ifftn(np.where(on, A, 0.0))))
    return out


def dns_grid_and_state(n, seed=1):
    """The fixture's start (`dns_start`, :120-137): the field of spectrum
    k^4 exp(-2 (k/1.5)^2) scaled to K = 3/2, as storage arrays."""
    from aeolus_b200 import regular_grid
    from aeolus_b200.inputs import embed
    g = regular_grid((n, n, n), (2 * np.pi,) * 3)
    u, v, w = random_field(n, lambda k: k ** 4 * np.exp(-2 * (k / KP) ** 2), seed)
    K = 0.5 * float(np.mean(u * u) + np.mean(v * v) + np.mean(w * w))
    s = np.sqrt(1.5 / K)
    return g, tuple(embed(g, a * s) for a in (u, v, w)) + (g.zeros(),)


def dns_nu(n):
    return NU48 * (48 / n) ** (4 / 3)


def _lap(a, h):
    return sum((np.roll(a, -1, ax) - 2 * a + np.roll(a, 1, ax)) for ax in range(3)) / (h * h)


def diagnostics(u, v, w, h, nu):
    """(K, eps, S, umax) of interior velocity arrays [k][j][i] on the uniform
    periodic grid of spacing h."""
    K = 0.5 * float(np.mean(u * u) + np.mean(v * v) + np.mean(w * w))
    eps = -nu * float(np.mean(u * _lap(u, h)) + np.mean(v * _lap(v, h)) + np.mean(w * _lap(w, h)))
    num = den = 0.0
    for a, ax in ((u, 2), (v, 1), (w, 0)):
        gdf = (np.roll(a, -1, ax) - a) / h
        g2 = gdf * gdf
        num += float(np.mean(g2 * gdf))
        den += float(np.mean(g2))
    S = (num / 3) / (den / 3) ** 1.5
    umax = max(float(np.abs(a).max()) for a in (u, v, w))
    return K, eps, S, umax


def run(sim, g, nu, t_end=2.0, cfl=0.5, max_steps=400):
    """Step `sim` (anything with get_field and step_rk3) as `dns_step!` does
    to t_end; returns the history arrays t, K, eps, S, budget_err, dts."""
    def diag():
        f = [sim.get_field(n)[g.interior] for n in ("u", "v", "w")]
        return diagnostics(*f, g.dx, nu)

    t = 0.0
    K, eps, S, umax = diag()
    hist = {"t": [0.0], "K": [K], "eps": [eps], "S": [S], "budget_err": [], "dt": []}
    for _ in range(max_steps):
        if t >= t_end - 1e-12:
            break
        dt = min(cfl * g.dx / umax, t_end - t)
        sim.step_rk3(dt, 1)
        t += dt
        K, eps, S, umax = diag()
        hist["t"].append(t)
        hist["K"].append(K)
        hist["eps"].append(eps)
        hist["S"].append(S)
        hist["dt"].append(dt)
        hist["budget_err"].append(-(hist["K"][-1] - hist["K"][-2]) / dt / (0.5 * (hist["eps"][-1] + hist["eps"][-2])) - 1)
    return {k: np.asarray(v) for k, v in hist.items()}


def kmax_eta(hist, n, nu):
    eta = (nu ** 3 / hist["eps"]) ** 0.25
    return float(np.min((n / 2) * eta))   # k_max = pi / dx = n / 2 on the 2 pi box
