"""TEST INFRASTRUCTURE ONLY: ctypes binding of the multigrid / MG-preconditioned
CG oracle (oracle/mgpcg.c), the checker of the library's cut-cell pressure
solve.  Arrays are interior-only numpy arrays indexed [k, j, i]."""
from __future__ import annotations

import ctypes as C

import numpy as np

from .oracle import load

_D = C.POINTER(C.c_double)

BCS = {"periodic": 0, "neumann": 1}
PRECONDITIONERS = {"identity": 0, "vcycle": 1}
STATUS = {0: "converged", 1: "maxit", 2: "breakdown", 3: "zero_rhs"}


class OcgParams(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
                ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
                ("bc_x", C.c_int32), ("bc_y", C.c_int32), ("bc_z", C.c_int32),
                ("tol", C.c_double), ("maxit", C.c_int32), ("nu1", C.c_int32), ("nu2", C.c_int32),
                ("coarse_sweeps", C.c_int32), ("min_size", C.c_int32), ("mg_cycles", C.c_int32),
                ("precond", C.c_int32)]


class OcgStats(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("status", C.c_int32),
                ("residual", C.c_double), ("bnorm", C.c_double), ("curvature", C.c_double)]


_bound = False


def _lib():
    global _bound
    L = load()
    if not _bound:
        L.ocg_create.restype = C.c_void_p
        L.ocg_create.argtypes = [C.POINTER(OcgParams), _D, _D, _D]
        L.ocg_destroy.argtypes = [C.c_void_p]
        L.ocg_nlevels.argtypes = [C.c_void_p]
        L.ocg_level_dims.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int32)]
        L.ocg_level_coeff.argtypes = [C.c_void_p, C.c_int, _D, _D, _D]
        for f in (L.ocg_apply, L.ocg_precondition):
            f.argtypes = [C.c_void_p, _D, _D]
        for f in (L.ocg_solve, L.ocg_mg_solve):
            f.argtypes = [C.c_void_p, _D, _D, C.POINTER(OcgStats)]
        _bound = True
    return L


def _p(a):
    return a.ctypes.data_as(_D)


class OracleMGPCG:
    """MGPreconditionedCG / MultigridPoissonSolver of the reference
    (src/Multigrid.jl:551-600, :893-967) on an nx x ny x nz grid."""

    def __init__(self, shape, spacing, coeffs=None, bc=("periodic", "periodic", "neumann"),
                 tol=1e-10, maxit=200, nu1=2, nu2=2, coarse_sweeps=50, min_size=4, mg_cycles=1,
                 precond="vcycle"):
        nx, ny, nz = shape
        self.shape = (nz, ny, nx)
        self.p = OcgParams(nx, ny, nz, *map(float, spacing), *(BCS[b] for b in bc), float(tol), int(maxit),
                           nu1, nu2, coarse_sweeps, min_size, mg_cycles, PRECONDITIONERS[precond])
        self._c = None
        if coeffs is not None:
            cx, cy, cz = (np.ascontiguousarray(c, dtype=np.float64) for c in coeffs)
            assert cx.shape == (nz, ny, nx + 1) and cy.shape == (nz, ny + 1, nx) and cz.shape == (nz + 1, ny, nx)
            self._c = (cx, cy, cz)
            h = _lib().ocg_create(C.byref(self.p), _p(cx), _p(cy), _p(cz))
        else:
            h = _lib().ocg_create(C.byref(self.p), None, None, None)
        if not h:
            raise ValueError("invalid multigrid parameters")
        self.h = C.c_void_p(h)

    def __del__(self):
        if getattr(self, "h", None):
            _lib().ocg_destroy(self.h)
            self.h = None

    @property
    def nlevels(self):
        return _lib().ocg_nlevels(self.h)

    def level_dims(self, lev):
        d = (C.c_int32 * 3)()
        _lib().ocg_level_dims(self.h, lev, d)
        return tuple(d)

    def level_coeff(self, lev):
        nx, ny, nz = self.level_dims(lev)
        cx, cy, cz = np.zeros((nz, ny, nx + 1)), np.zeros((nz, ny + 1, nx)), np.zeros((nz + 1, ny, nx))
        if _lib().ocg_level_coeff(self.h, lev, _p(cx), _p(cy), _p(cz)):
            raise ValueError("no coefficients")
        return cx, cy, cz

    def _arr(self, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        assert a.shape == self.shape
        return a

    def apply(self, x):
        x = self._arr(x)
        out = np.zeros(self.shape)
        _lib().ocg_apply(self.h, _p(x), _p(out))
        return out

    def precondition(self, r):
        r = self._arr(r)
        z = np.zeros(self.shape)
        _lib().ocg_precondition(self.h, _p(r), _p(z))
        return z

    def _run(self, f, b):
        b = self._arr(b)
        x = np.zeros(self.shape)
        st = OcgStats()
        f(self.h, _p(b), _p(x), C.byref(st))
        return x, {"iterations": st.iterations, "status": STATUS[st.status], "residual": st.residual,
                   "bnorm": st.bnorm, "relative_residual": 0.0 if st.bnorm == 0 else st.residual / st.bnorm,
                   "curvature": st.curvature}

    def solve(self, b):
        """solve!(p, source, ::MGPreconditionedCG) -> (x, stats)"""
        return self._run(_lib().ocg_solve, b)

    def mg_solve(self, b):
        """mg_solve!(solver, x, b) -> (x, stats); stats["residual"] is relative"""
        x, st = self._run(_lib().ocg_mg_solve, b)
        st["relative_residual"] = st["residual"]
        return x, st
