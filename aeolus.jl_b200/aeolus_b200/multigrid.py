"""MGPreconditionedCG / MultigridPoissonSolver on the GPU: the host mirror of
the reference's solver objects (src/Multigrid.jl:531-967) over the C ABI of
include/aeolus_b200_mgpcg.h.

    s = MGPreconditionedCG((nx, ny, nz), (dx, dy, dz), coeffs=(cx, cy, cz),
                           bc=("periodic", "periodic", "neumann"), tol=1e-10)
    x, stats = s.solve(b)          # solve!(p, source, ::MGPreconditionedCG)
    x, stats = s.mg_solve(b)       # mg_solve!(solver, x, b)

Arrays are interior-only numpy arrays indexed [k, j, i] (x fastest); face
coefficients cx (nz, ny, nx+1), cy (nz, ny+1, nx), cz (nz+1, ny, nx).
There is no CPU fallback: without the CUDA library construction raises.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L

BCS = {"periodic": 0, "neumann": 1}
PRECONDITIONERS = {"identity": 0, "vcycle": 1, "jacobi": 3}   # "learned": see MGPreconditionedCG.set_learned
PRECISIONS = {"fp64": 0, "fp32_mixed": 1}
STATUS = {0: "converged", 1: "maxit", 2: "breakdown", 3: "zero_rhs"}

_D = C.POINTER(C.c_double)


def _p(a):
    return a.ctypes.data_as(_D)


class MGPreconditionedCG:
    """CG preconditioned by `mg_cycles` = 1 V-cycle (the reference's
    MGPreconditionedCG).  precision "fp32_mixed" runs the cycle in FP32 with
    the Krylov vectors, the operator and the reductions in FP64;
    flexible=True uses the Polak-Ribiere beta (default for fp32_mixed)."""

    def __init__(self, shape, spacing, coeffs=None, bc=("periodic", "periodic", "neumann"), tol=1e-10,
                 maxit=200, nu1=2, nu2=2, coarse_sweeps=50, min_size=4, precision="fp64",
                 precond="vcycle", flexible=None, device=0):
        lib = L.load()
        nx, ny, nz = (int(v) for v in shape)
        self.shape = (nz, ny, nx)
        if flexible is None:
            flexible = precision != "fp64"
        if precision not in PRECISIONS:
            raise ValueError(f"unknown precision {precision!r}")
        if precond not in PRECONDITIONERS:
            raise ValueError(f"unknown preconditioner {precond!r}")
        try:
            bcs = [BCS[b] for b in bc]
        except KeyError as e:
            raise ValueError(f"unsupported BC {e} (use periodic or neumann)") from None
        self.cfg = L.AeoMgConfig(nx, ny, nz, *map(float, spacing), *bcs, PRECISIONS[precision],
                                 PRECONDITIONERS[precond], int(bool(flexible)), float(tol), int(maxit), int(nu1),
                                 int(nu2), int(coarse_sweeps), int(min_size), int(device))
        h = C.c_void_p()
        if coeffs is not None:
            cx, cy, cz = (np.ascontiguousarray(c, dtype=np.float64) for c in coeffs)
            if cx.shape != (nz, ny, nx + 1) or cy.shape != (nz, ny + 1, nx) or cz.shape != (nz + 1, ny, nx):
                raise ValueError("face coefficients must be (nz, ny, nx+1), (nz, ny+1, nx), (nz+1, ny, nx)")
            L.check(lib.aeo_mg_create(C.byref(self.cfg), _p(cx), _p(cy), _p(cz), C.byref(h)), None, mg=True)
        else:
            L.check(lib.aeo_mg_create(C.byref(self.cfg), None, None, None, C.byref(h)), None, mg=True)
        self._h = h
        self.last_stats = None

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            L.load().aeo_mg_destroy(h)
            self._h = None

    def _chk(self, s):
        L.check(s, self._h, mg=True)

    @property
    def nlevels(self) -> int:
        """mg_level_count (src/Multigrid.jl:670)."""
        n = C.c_int32()
        self._chk(L.load().aeo_mg_levels(self._h, C.byref(n), None))
        return n.value

    def level_dims(self):
        n = self.nlevels
        d = (C.c_int32 * (3 * n))()
        self._chk(L.load().aeo_mg_levels(self._h, None, d))
        return [tuple(d[3 * l:3 * l + 3]) for l in range(n)]

    def _arr(self, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        if a.shape != self.shape:
            raise ValueError(f"array shape {a.shape} != {self.shape}")
        return a

    @staticmethod
    def _stats(st, relative):
        return {"iterations": st.iterations, "status": STATUS[st.status], "residual": st.residual,
                "bnorm": st.bnorm,
                "relative_residual": st.residual if relative else (0.0 if st.bnorm == 0 else st.residual / st.bnorm),
                "curvature": st.curvature, "fallback_at": st.fallback_at}

    def solve(self, b, out=None):
        """x = A^-1 b by MG-preconditioned CG (solve!, src/Multigrid.jl:955-967).
        `out`: an optional C-contiguous float64 array (e.g. pinned) for x."""
        b = self._arr(b)
        x = np.empty(self.shape) if out is None else out
        if x.shape != self.shape or x.dtype != np.float64 or not x.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous float64 array of the grid's shape")
        st = L.AeoMgStats()
        self._chk(L.load().aeo_mg_solve(self._h, _p(b), _p(x), C.byref(st)))
        self.last_stats = self._stats(st, False)
        return x, self.last_stats

    def set_learned(self, net, stagnation=0.9):
        """Precondition flexible CG with the learned U-Net `net` (an
        aeolus_b200.unet.UNet of this grid, its mask set); None restores the
        V-cycle.  A solve falls back to the V-cycle for its remaining
        iterations after two iterations in a row whose residual fell by less
        than `stagnation`."""
        self._chk(L.load().aeo_mg_set_learned(self._h, net.handle if net is not None else None, float(stagnation)))
        self._net = net

    def solve_harvest(self, b, cap=16):
        """solve() that also returns the residuals r_k and iterates x_k of the
        CG iterations: (x, stats, [(r_k, x - x_k)]), residual -> error pairs."""
        b = self._arr(b)
        x = np.empty(self.shape)
        rh = np.empty((cap,) + self.shape)
        xh = np.empty((cap,) + self.shape)
        cnt = C.c_int32()
        st = L.AeoMgStats()
        self._chk(L.load().aeo_mg_solve_harvest(self._h, _p(b), _p(x), C.byref(st), _p(rh), _p(xh), int(cap),
                                                C.byref(cnt)))
        self.last_stats = self._stats(st, False)
        return x, self.last_stats, [(rh[k], x - xh[k]) for k in range(cnt.value)]

    def solve_device(self, b_ptr: int, x_ptr: int):
        """The same on FP64 device arrays (raw device pointers)."""
        st = L.AeoMgStats()
        self._chk(L.load().aeo_mg_solve_device(self._h, C.c_void_p(b_ptr), C.c_void_p(x_ptr), C.byref(st)))
        self.last_stats = self._stats(st, False)
        return self.last_stats

    def mg_solve(self, b):
        """Multigrid cycles until the relative residual is below tol (mg_solve!)."""
        b = self._arr(b)
        x = np.empty(self.shape)
        st = L.AeoMgStats()
        self._chk(L.load().aeo_mg_vcycle_solve(self._h, _p(b), _p(x), C.byref(st)))
        self.last_stats = self._stats(st, True)
        return x, self.last_stats

    def apply(self, x):
        """A x (_apply_fine!, src/Multigrid.jl:911-919)."""
        x = self._arr(x)
        out = np.empty(self.shape)
        self._chk(L.load().aeo_mg_apply(self._h, _p(x), _p(out)))
        return out

    def precondition(self, r):
        """z = M r, one V-cycle (_mg_precond!, src/Multigrid.jl:922-932)."""
        r = self._arr(r)
        z = np.empty(self.shape)
        self._chk(L.load().aeo_mg_precondition(self._h, _p(r), _p(z)))
        return z

    def profile(self, what: str, reps: int = 20) -> float:
        """Mean device ms of one part: "solve", "rbgs" (one finest colour
        pass), "apply" (operator + p.Ap), "vcycle", "coarsest" (the
        coarsest-level sweeps), "restrict" (finest residual restriction),
        "sweep" (one whole finest red-black sweep as the cycle runs it)."""
        code = {"solve": 0, "rbgs": 1, "apply": 2, "vcycle": 3, "coarsest": 4, "restrict": 5, "sweep": 6}[what]
        ms = C.c_double()
        self._chk(L.load().aeo_mg_profile(self._h, code, int(reps), C.byref(ms)))
        return ms.value

    @property
    def launches_per_iteration(self) -> int:
        return L.load().aeo_mg_launches_per_iteration(self._h)


def MultigridPoissonSolver(shape, spacing, **kw):
    """The standalone multigrid solver: `mg_solve` of an MGPreconditionedCG
    handle (the same hierarchy, src/Multigrid.jl:551-600)."""
    kw.setdefault("maxit", 50)
    return MGPreconditionedCG(shape, spacing, **kw)
