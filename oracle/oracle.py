"""TEST INFRASTRUCTURE ONLY: ctypes binding of the oracle (oracle/aeolus_oracle.c).

The oracle is a CPU FP64 restatement of the reference's dynamical-core step;
tests, `__graft_entry__.smoke()` and bench.py's CPU-baseline leg use it as the
checker.  It takes the same `CoreSpec` as the product library.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "libaeolus_oracle.so")

_D = C.POINTER(C.c_double)


class OcParams(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("hx", C.c_int32), ("hy", C.c_int32), ("hz", C.c_int32),
        ("lx", C.c_double), ("ly", C.c_double), ("lz", C.c_double),
        ("x0", C.c_double), ("y0", C.c_double), ("z0", C.c_double),
        ("stretched", C.c_int32), ("bc_x", C.c_int32), ("bc_y", C.c_int32), ("bc_z", C.c_int32),
        ("core", C.c_int32), ("advection", C.c_int32), ("solver", C.c_int32),
        ("nu", C.c_double), ("theta0", C.c_double), ("g", C.c_double), ("f_coriolis", C.c_double),
        ("c_s", C.c_double), ("pr_t", C.c_double),
        ("flux_bot", C.c_double), ("flux_top", C.c_double), ("sponge_alpha", C.c_double),
        ("sponge_zstart", C.c_double), ("sgs_model", C.c_int32),
    ]


class OcCfl(C.Structure):
    _fields_ = [("c_adv", C.c_double), ("c_diff", C.c_double), ("c_buoy", C.c_double), ("c_cor", C.c_double),
                ("dt_min", C.c_double), ("dt_max", C.c_double), ("growth", C.c_double)]


def _cfl(c):
    return OcCfl(c.C_advective, c.C_diffusive, c.C_buoyancy, c.C_coriolis, c.dt_min, c.dt_max, c.growth_max)


_lib = None


def build():
    r = subprocess.run(["make", "-C", _HERE], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stdout}\n{r.stderr}")
    return LIB_PATH


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        build()
    lib = C.CDLL(LIB_PATH)
    P = C.c_void_p
    lib.oc_create.argtypes = [C.POINTER(OcParams), _D, _D, _D, _D]
    lib.oc_create.restype = P
    lib.oc_destroy.argtypes = [P]
    lib.oc_storage_size.argtypes = [P]
    lib.oc_storage_size.restype = C.c_int64
    lib.oc_set_field.argtypes = [P, C.c_int, _D]
    lib.oc_get_field.argtypes = [P, C.c_int, _D]
    lib.oc_fill_state_halos.argtypes = [P]
    lib.oc_step_rk3.argtypes = [P, C.c_double, C.c_int]
    lib.oc_step_euler.argtypes = [P, C.c_double, C.c_int]
    lib.oc_project.argtypes = [P]
    lib.oc_adaptive_dt.argtypes = [P, C.POINTER(OcCfl), C.c_double, C.POINTER(C.c_int)]
    lib.oc_adaptive_dt.restype = C.c_double
    lib.oc_step_adaptive.argtypes = [P, C.POINTER(OcCfl), C.c_int, C.POINTER(C.c_double), _D]
    lib.oc_tendencies.argtypes = [P, _D, _D, _D, _D]
    lib.oc_pressure_solve.argtypes = [P, _D, _D]
    lib.oc_apply_poisson_operator.argtypes = [P, _D, _D]
    lib.oc_kinetic_energy.argtypes = [P]
    lib.oc_kinetic_energy.restype = C.c_double
    lib.oc_max_divergence.argtypes = [P]
    lib.oc_max_divergence.restype = C.c_double
    lib.oc_set_threads.argtypes = [C.c_int]
    lib.oc_set_ibm.argtypes = [P, C.c_void_p, C.c_double]
    lib.oc_advect_positive.argtypes = [P, _D, _D, _D, _D, _D, C.c_double, C.c_int, C.c_int]
    lib.oc_set_apertures.argtypes = [P, _D, _D, _D, C.c_double, C.c_int]
    lib.oc_set_open.argtypes = [P, C.c_int, C.c_int, _D, _D, C.POINTER(C.c_int)]
    lib.oc_set_open_outflow.argtypes = [P, C.POINTER(C.c_int), C.c_int, _D, _D, _D, _D]
    lib.oc_open_ledger.argtypes = [P, _D]
    lib.oc_open_ledger.restype = None
    lib.oc_get_open_planes.argtypes = [P, _D, _D]
    lib.oc_get_open_planes.restype = None
    lib.oc_set_open_planes.argtypes = [P, _D, _D]
    lib.oc_set_open_planes.restype = C.c_int
    lib.oc_open_history.argtypes = [P, _D, _D, _D, C.c_int]
    lib.oc_open_history.restype = C.c_int
    lib.oc_set_sgs_buoyancy.argtypes = [P, _D]
    lib.oc_set_lagrangian.argtypes = [P, C.c_double, C.c_double, C.c_double]
    lib.oc_set_tke.argtypes = [P, C.c_double, C.c_double, C.c_double, C.c_int]
    lib.oc_get_sgs_state.argtypes = [P, _D]
    lib.oc_set_sgs_state.argtypes = [P, _D]
    lib.oc_pcg_stats.argtypes = [P, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_double),
                                 C.POINTER(C.c_double)]
    lib.oc_philox4x32.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
    lib.oc_uniform_fill.argtypes = [C.c_uint64, C.c_uint32, C.c_int64, C.c_double, _D]
    _lib = lib
    return lib


FIELD_IDS = {"u": 0, "v": 1, "w": 2, "theta": 3, "p": 4, "nut": 5, "phi": 6, "kt": 7}
_ADV = {"centred": 0, "weno_js5": 1, "weno_z5": 2}
_SOLV = {"fft": 0, "column": 1, "pcg": 2}
_PCG_STATUS = {0: "converged", 1: "maxit", 2: "breakdown", 3: "zero_rhs"}
_CORE = {"boussinesq": 0, "anelastic": 1}


def _p(a):
    return None if a is None else a.ctypes.data_as(_D)


def set_threads(n: int):
    load().oc_set_threads(int(n))


def philox4x32(ctr, key):
    lib = load()
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib.oc_philox4x32(c, k, o)
    return tuple(int(x) for x in o)


def uniform_fill(seed: int, stream: int, n: int, amp: float) -> np.ndarray:
    out = np.empty(n)
    load().oc_uniform_fill(seed, stream, n, amp, _p(out))
    return out


class OracleSimulation:
    """The oracle's domain: same CoreSpec and storage-array interface as aeolus_b200.Simulation."""

    def __init__(self, spec):
        lib = load()
        g = spec.grid
        p = OcParams()
        p.nx, p.ny, p.nz = g.size
        p.hx, p.hy, p.hz = g.halo
        p.lx, p.ly, p.lz = g.extent
        p.x0, p.y0, p.z0 = g.origin
        p.stretched = 1 if g.stretched else 0
        p.bc_x = p.bc_y = 0
        p.bc_z = 0 if g.bc_z == "periodic" else 1
        p.core = _CORE[spec.core]
        p.advection = _ADV[spec.advection]
        p.solver = _SOLV[spec.solver]
        p.nu, p.theta0, p.g, p.f_coriolis = spec.nu, spec.theta0, spec.g, spec.f_coriolis
        p.c_s, p.pr_t = spec.c_s, spec.pr_t
        p.flux_bot, p.flux_top = spec.flux_bot, spec.flux_top
        p.sponge_alpha, p.sponge_zstart = spec.sponge_alpha, spec.sponge_zstart
        p.sgs_model = {"smagorinsky": 0, "vreman": 1, "sigma": 2, "amd": 3, "dynamic": 4, "lagrangian": 6, "tke": 7}[spec.sgs]
        if spec.sgs == "dynamic" and getattr(spec, "averaging", "plane") == "local":
            p.sgs_model = 5
        self._keep = [g.zf, spec.wc, spec.wf, spec.thf]
        h = lib.oc_create(C.byref(p), _p(g.zf), _p(spec.wc), _p(spec.wf), _p(spec.thf))
        if not h:
            raise ValueError("oracle: unsupported configuration")
        self._h = h
        self._lib = lib
        self.spec = spec
        self.grid = g
        if spec.sgs == "amd" and spec.c_s != 0 and spec.core == "anelastic":
            self._bg = np.ascontiguousarray(spec.g / spec.thc, dtype=np.float64)
            self._lib.oc_set_sgs_buoyancy(self._h, _p(self._bg))
        if spec.sgs == "lagrangian" and spec.c_s != 0:
            mt = spec.lag_memory_time
            assert self._lib.oc_set_lagrangian(self._h, spec.lag_c0, spec.lag_theta, 0.0 if mt is None else mt) == 0

        if spec.sgs == "tke" and spec.c_s != 0:
            assert self._lib.oc_set_tke(self._h, spec.tke_c_eps0, spec.tke_c_eps1, spec.tke_c_l,
                                        1 if spec.tke_dissipation == "exact" else 0) == 0
            if spec.tke_e0:
                self.set_sgs_state(np.full((g.nz, g.ny, g.nx), float(spec.tke_e0)))

    def sgs_state(self):
        """The Lagrangian closure's memory: (I_LM, I_MM, U, V, W) as (nz, ny, nx)
        arrays and the initialised flag; the TKE closure's: e (nz, ny, nx)."""
        g = self.grid
        n = g.nx * g.ny * g.nz
        if self.spec.sgs == "tke":
            out = np.empty(n)
            assert self._lib.oc_get_sgs_state(self._h, _p(out)) == 0
            return out.reshape(g.nz, g.ny, g.nx)
        out = np.empty(5 * n + 1)
        assert self._lib.oc_get_sgs_state(self._h, _p(out)) == 0
        arrs = tuple(out[f * n:(f + 1) * n].reshape(g.nz, g.ny, g.nx).copy() for f in range(5))
        return arrs + (bool(out[5 * n]),)

    def set_sgs_state(self, state):
        if self.spec.sgs == "tke":
            a = np.ascontiguousarray(state, dtype=np.float64).ravel()
            assert self._lib.oc_set_sgs_state(self._h, _p(a)) == 0
            return
        a = np.concatenate([np.ascontiguousarray(x, dtype=np.float64).ravel() for x in state[:5]] +
                           [np.array([1.0 if state[5] else 0.0])])
        assert self._lib.oc_set_sgs_state(self._h, _p(a)) == 0

    def close(self):
        if getattr(self, "_h", None):
            self._lib.oc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_field(self, name, data):
        a = np.ascontiguousarray(data, dtype=np.float64)
        assert a.shape == self.grid.storage_shape
        assert self._lib.oc_set_field(self._h, FIELD_IDS[name], _p(a)) == 0

    def get_field(self, name):
        out = np.empty(self.grid.storage_shape)
        assert self._lib.oc_get_field(self._h, FIELD_IDS[name], _p(out)) == 0
        return out

    def set_state(self, u, v, w, theta):
        for n, a in zip(("u", "v", "w", "theta"), (u, v, w, theta)):
            self.set_field(n, a)

    def get_state(self):
        return tuple(self.get_field(n) for n in ("u", "v", "w", "theta"))

    def fill_halos(self):
        self._lib.oc_fill_state_halos(self._h)

    def step_rk3(self, dt, nsteps=1):
        assert self._lib.oc_step_rk3(self._h, float(dt), int(nsteps)) == 0

    def step(self, dt, nsteps=1):
        assert self._lib.oc_step_euler(self._h, float(dt), int(nsteps)) == 0

    def adaptive_dt(self, constraints, dt_prev=None):
        lim = C.c_int()
        dt = self._lib.oc_adaptive_dt(self._h, C.byref(_cfl(constraints)), float(dt_prev or 0.0), C.byref(lim))
        return dt, lim.value

    def step_adaptive(self, constraints, nsteps=1, dt_prev=None):
        d = C.c_double(float(dt_prev or 0.0))
        dts = np.empty(nsteps)
        self._lib.oc_step_adaptive(self._h, C.byref(_cfl(constraints)), int(nsteps), C.byref(d), _p(dts))
        return dts

    def project(self):
        assert self._lib.oc_project(self._h) == 0

    def tendencies(self):
        outs = [np.empty(self.grid.storage_shape) for _ in range(4)]
        self._lib.oc_tendencies(self._h, *[_p(o) for o in outs])
        return outs

    def pressure_solve(self, src):
        g = self.grid
        s = np.ascontiguousarray(src, dtype=np.float64)
        assert s.shape == (g.nz, g.ny, g.nx)
        out = np.empty_like(s)
        self._lib.oc_pressure_solve(self._h, _p(s), _p(out))
        return out

    def apply_poisson_operator(self, phi):
        p = np.ascontiguousarray(phi, dtype=np.float64)
        out = np.empty_like(p)
        self._lib.oc_apply_poisson_operator(self._h, _p(p), _p(out))
        return out

    def set_ibm(self, mask=None, tau=0.0):
        """The implicit IBM correction after every predictor: a storage-shaped
        solid mask (None: off) and tau (0: blocked faces zeroed)."""
        if mask is None:
            ptr = None
        else:
            m = np.ascontiguousarray(mask, dtype=np.uint8)
            assert m.shape == self.grid.storage_shape
            self._ibm = m
            ptr = m.ctypes.data_as(C.c_void_p)
        if self._lib.oc_set_ibm(self._h, ptr, float(tau)) != 0:
            raise ValueError("oracle: set_ibm rejected (tau < 0, or the PCG solver)")

    def set_pcg(self, apertures=None, tol=1e-8, maxit=200):
        """solver = "pcg": the face apertures (ax, ay, az) in the interior face
        layout (None: every face open) and the CG tolerance and cap."""
        if apertures is None:
            ptrs = (None, None, None)
        else:
            g = self.grid
            nx, ny, nz = g.size
            a = [np.ascontiguousarray(x, dtype=np.float64) for x in apertures]
            assert a[0].shape == (nz, ny, nx + 1) and a[1].shape == (nz, ny + 1, nx) and a[2].shape == (nz + 1, ny, nx)
            self._ap = a
            ptrs = tuple(_p(x) for x in a)
        if self._lib.oc_set_apertures(self._h, *ptrs, float(tol), int(maxit)) != 0:
            raise ValueError("oracle: set_pcg rejected (solver, tolerance or apertures)")

    def set_open_boundaries(self, obc=None):
        """Open lateral faces from an OpenBoundarySet (None closes them)."""
        if obc is None:
            if self._lib.oc_set_open(self._h, 0, 0, None, None, None) != 0:
                raise ValueError("oracle: set_open rejected")
            self._open = None
            return
        xp, yp, modes = obc.packed()
        m = np.ascontiguousarray(modes, dtype=np.int32)
        self._open = (xp, yp, m)
        if self._lib.oc_set_open(self._h, int(obc.open_x), int(obc.open_y), _p(xp), _p(yp),
                                 m.ctypes.data_as(C.POINTER(C.c_int))) != 0:
            raise ValueError("oracle: set_open rejected (needs the PCG solver on the uniform Boussinesq core, "
                             "walls in z, a static SGS closure if any)")
        rad = np.ascontiguousarray(obc.radiating, dtype=np.int32)
        xd, yd, _ = obc.packed(raw=True)
        xf, yf = obc.face_weights()
        self._open_raw = (rad, xd, yd, xf, yf)
        if self._lib.oc_set_open_outflow(self._h, rad.ctypes.data_as(C.POINTER(C.c_int)), int(obc.correction_code),
                                         _p(xd), _p(yd), _p(xf), _p(yf)) != 0:
            raise ValueError("oracle: set_open_outflow rejected")

    def open_planes(self):
        xp, yp = (np.zeros_like(a) for a in self._open_raw[1:3])
        self._lib.oc_get_open_planes(self._h, _p(xp), _p(yp))
        return xp, yp

    def open_checkpoint(self):
        """The planes and, on a radiating set, the :orlanski history
        (open_boundary_checkpoint, open_boundary.jl:1282-1305); None without
        open faces."""
        if getattr(self, "_open", None) is None:
            return None
        xp, yp = self.open_planes()
        out = {"planes_x": xp, "planes_y": yp}
        if self._open_raw[0].any():
            NZ, NY, NX = self.grid.storage_shape
            hx, hy, sc = np.zeros((4, 2, NZ, NY)), np.zeros((4, 2, NZ, NX)), np.zeros(2)
            assert self._lib.oc_open_history(self._h, _p(hx), _p(hy), _p(sc), 0) == 0
            out.update({"hist_x": hx, "hist_y": hy, "hist_set": float(sc[0]), "last_dt": float(sc[1])})
        return out

    def restore_open_checkpoint(self, state):
        """Copy an open_checkpoint back (restore_open_boundary_checkpoint!,
        open_boundary.jl:1307-1350) into faces built as the checkpointed ones."""
        if state is None:
            return
        if getattr(self, "_open", None) is None:
            raise ValueError("restore: the checkpoint has open faces, the domain none")
        if state["planes_x"].shape != self._open[0].shape or state["planes_y"].shape != self._open[1].shape:
            raise ValueError("restore: the open faces are built differently from the checkpoint's")
        if ("hist_x" in state) != bool(self._open_raw[0].any()):
            raise ValueError("restore: the radiating faces differ from the checkpoint's")
        xp, yp = (np.ascontiguousarray(state[k], dtype=np.float64) for k in ("planes_x", "planes_y"))
        assert self._lib.oc_set_open_planes(self._h, _p(xp), _p(yp)) == 0
        if "hist_x" in state:
            hx, hy = (np.ascontiguousarray(state[k], dtype=np.float64) for k in ("hist_x", "hist_y"))
            sc = np.array([state["hist_set"], state["last_dt"]])
            assert self._lib.oc_open_history(self._h, _p(hx), _p(hy), _p(sc), 1) == 0

    def open_ledger(self):
        out = np.zeros(3)
        self._lib.oc_open_ledger(self._h, _p(out))
        return {"Q": out[0], "residual": out[1], "delta": out[2]}

    def pcg_stats(self):
        it, stt = C.c_int(), C.c_int()
        r, b = C.c_double(), C.c_double()
        assert self._lib.oc_pcg_stats(self._h, C.byref(it), C.byref(stt), C.byref(r), C.byref(b)) == 0
        return {"iterations": it.value, "status": _PCG_STATUS[stt.value], "residual": r.value, "bnorm": b.value,
                "relative_residual": 0.0 if b.value == 0 else r.value / b.value}

    def advect_positive(self, u, v, w, phi, dt, scheme="weno_z5", tend=None, accumulate=True):
        """advect_positive!: tend (a copy, zeros if None) with -div(u phi)
        added (accumulate) or written, the positivity limiter applied; storage
        arrays with filled halos."""
        g = self.grid
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (u, v, w, phi)]
        for a in arrs:
            assert a.shape == g.storage_shape
        out = np.zeros(g.storage_shape) if tend is None else np.array(tend, dtype=np.float64, copy=True)
        rc = self._lib.oc_advect_positive(self._h, *[_p(a) for a in arrs], _p(out), float(dt), _ADV[scheme],
                                          int(bool(accumulate)))
        if rc != 0:
            raise ValueError("oracle: advect_positive needs a uniform grid, halo >= 3 and a WENO scheme")
        return out

    def kinetic_energy(self):
        return self._lib.oc_kinetic_energy(self._h)

    def max_divergence(self):
        return self._lib.oc_max_divergence(self._h)
