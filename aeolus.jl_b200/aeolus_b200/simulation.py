"""The host-side mirror of the reference's step-core interface.

`Simulation` holds one domain on a B200 through the C-ABI.  Its methods are
the reference's operations on a `BoussinesqSimulation`
(src/Simulations.jl:168-246) or a sound-proof simulation
(src/Anelastic.jl:1559): `step_rk3` (`step_rk3!`, src/Simulations.jl:843),
`step` (`step!`, :481), `kinetic_energy` (:992), `max_divergence` (:1045)
and the pressure-solver seam `pressure_solve` (`solve!`,
src/PressureSolvers.jl:41-80).  Fields move as the reference's `Field.data`
storage arrays (numpy shape (Nz+2Hz, Ny+2Hy, Nx+2Hx), Float64).

Errors follow the reference: a bad argument raises ValueError (ArgumentError),
a non-finite state after a step raises NumericalFailure.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _lib
from .grids import PERIODIC, WALL, Grid
from .reference_state import anelastic_profiles
from .spec import ADVECTION, CORES, FIELDS, PRECISIONS, SGS_MODELS, SOLVERS, CoreSpec, sgs_buoyancy_levels, sgs_model_code

_D = C.POINTER(C.c_double)


def _ptr(a: Optional[np.ndarray]):
    if a is None:
        return None
    return a.ctypes.data_as(_D)


class CFLConstraints:
    """`CFLConstraints` (src/TimeIntegration.jl:127-153) with the guard limits
    of `step_adaptive!` (divergence_tol, max_velocity, max_retries)."""

    def __init__(self, C_advective=0.5, C_diffusive=0.25, C_buoyancy=0.5, C_coriolis=0.5, dt_min=1e-8,
                 dt_max=float("inf"), growth_max=1.1, divergence_tol=1e-6, max_velocity=float("inf"), max_retries=3):
        if not (C_advective > 0 and C_diffusive > 0 and C_buoyancy > 0 and C_coriolis > 0):
            raise ValueError("CFL numbers must be > 0")
        if not (0 < dt_min <= dt_max):
            raise ValueError("need 0 < dt_min <= dt_max")
        if not growth_max >= 1:
            raise ValueError("growth_max must be >= 1")
        self.__dict__.update(locals())
        del self.__dict__["self"]

    def to_c(self):
        return _lib.AeoCfl(self.C_advective, self.C_diffusive, self.C_buoyancy, self.C_coriolis, self.dt_min,
                           self.dt_max, self.growth_max, self.divergence_tol, self.max_velocity, self.max_retries)


def _stats(st) -> dict:
    return {"dt": st.dt, "t_advanced": st.t_advanced, "limiter": _lib.LIMITERS[st.limiter], "retries": st.retries,
            "advective_rate": st.advective_rate, "nut_max": st.nut_max, "N": st.brunt_vaisala,
            "max_divergence": st.max_divergence, "max_speed": st.max_speed}


class Simulation:
    def __init__(self, spec: CoreSpec, device: int = 0):
        self.spec = spec
        self.grid = spec.grid
        lib = _lib.load()
        g = spec.grid
        cfg = _lib.AeoConfig()
        cfg.nx, cfg.ny, cfg.nz = g.size
        cfg.hx, cfg.hy, cfg.hz = g.halo
        cfg.lx, cfg.ly, cfg.lz = g.extent
        cfg.x0, cfg.y0, cfg.z0 = g.origin
        cfg.bc_x = cfg.bc_y = 0
        cfg.bc_z = 0 if g.bc_z == PERIODIC else 1
        cfg.stretched = 1 if g.stretched else 0
        cfg.core = CORES[spec.core]
        cfg.advection = ADVECTION[spec.advection]
        cfg.sgs_model = sgs_model_code(spec)
        cfg.solver = SOLVERS[spec.solver]
        cfg.precision = PRECISIONS[spec.precision]
        cfg.nu, cfg.theta0, cfg.g, cfg.f_coriolis = spec.nu, spec.theta0, spec.g, spec.f_coriolis
        cfg.c_s, cfg.pr_t = spec.c_s, spec.pr_t
        cfg.flux_bot, cfg.flux_top = spec.flux_bot, spec.flux_top
        cfg.sponge_alpha, cfg.sponge_zstart = spec.sponge_alpha, spec.sponge_zstart
        cfg.device = device
        self._keep = [spec.grid.zf, spec.wc, spec.wf, spec.thf]
        h = C.c_void_p()
        st = lib.aeo_create(C.byref(cfg), _ptr(g.zf), _ptr(spec.wc), _ptr(spec.wf), _ptr(spec.thf), C.byref(h))
        _lib.check(st, None)
        self._h = h
        self._lib = lib
        bg = sgs_buoyancy_levels(spec)
        if bg is not None:
            bg = np.ascontiguousarray(bg, dtype=np.float64)
            _lib.check(lib.aeo_set_sgs_buoyancy(h, _ptr(bg)), h)
        if spec.sgs == "lagrangian" and spec.c_s != 0:
            mt = spec.lag_memory_time
            _lib.check(lib.aeo_set_lagrangian(h, spec.lag_c0, spec.lag_theta, 0.0 if mt is None else mt), h)
        if spec.sgs == "tke" and spec.c_s != 0:
            _lib.check(lib.aeo_set_tke(h, spec.tke_c_eps0, spec.tke_c_eps1, spec.tke_c_l,
                                       1 if spec.tke_dissipation == "exact" else 0), h)
            if spec.tke_e0:
                self.set_sgs_state(np.full((g.nz, g.ny, g.nx), float(spec.tke_e0)))

    # ---- lifecycle ------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            self._lib.aeo_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self):
        return self._h

    # ---- the closure's memory (sgs_state / restore_sgs_state!) -----------------
    def sgs_state(self):
        """The Lagrangian closure's committed memory: (I_LM, I_MM, U, V, W) as
        (nz, ny, nx) arrays and the initialised flag
        (src/operators/lagrangian_sgs.jl:372-381)."""
        g = self.grid
        n = g.nx * g.ny * g.nz
        if self.spec.sgs == "tke":       # e on the interior
            out = np.empty(n)
            _lib.check(self._lib.aeo_get_sgs_state(self._h, _ptr(out)), self._h)
            return out.reshape(g.nz, g.ny, g.nx)
        out = np.empty(5 * n + 1)
        _lib.check(self._lib.aeo_get_sgs_state(self._h, _ptr(out)), self._h)
        return tuple(out[f * n:(f + 1) * n].reshape(g.nz, g.ny, g.nx).copy() for f in range(5)) + (bool(out[5 * n]),)

    def set_sgs_state(self, state):
        g = self.grid
        if self.spec.sgs == "tke":
            a = np.ascontiguousarray(state, dtype=np.float64)
            if a.shape != (g.nz, g.ny, g.nx):
                raise ValueError(f"sgs state: e of shape {(g.nz, g.ny, g.nx)} expected")
            _lib.check(self._lib.aeo_set_sgs_state(self._h, _ptr(a)), self._h)
            return
        arrs = [np.ascontiguousarray(x, dtype=np.float64) for x in state[:5]]
        if any(a.shape != (g.nz, g.ny, g.nx) for a in arrs):
            raise ValueError(f"sgs state: five {(g.nz, g.ny, g.nx)} arrays and the initialised flag expected")
        a = np.concatenate([x.ravel() for x in arrs] + [np.array([1.0 if state[5] else 0.0])])
        _lib.check(self._lib.aeo_set_sgs_state(self._h, _ptr(a)), self._h)

    # ---- fields ---------------------------------------------------------------
    def set_field(self, name: str, data: np.ndarray):
        a = np.ascontiguousarray(data, dtype=np.float64)
        if a.shape != self.grid.storage_shape:
            raise ValueError(f"{name}: expected storage shape {self.grid.storage_shape}, got {a.shape}")
        _lib.check(self._lib.aeo_set_field(self._h, FIELDS[name], _ptr(a)), self._h)

    def get_field(self, name: str, out: Optional[np.ndarray] = None) -> np.ndarray:
        if out is None:
            out = np.empty(self.grid.storage_shape)
        _lib.check(self._lib.aeo_get_field(self._h, FIELDS[name], _ptr(out)), self._h)
        return out

    def set_field_f32(self, name: str, data: np.ndarray):
        """set_field from an FP32 host array (half the bytes)."""
        a = np.ascontiguousarray(data, dtype=np.float32)
        if a.shape != self.grid.storage_shape:
            raise ValueError(f"{name}: expected storage shape {self.grid.storage_shape}, got {a.shape}")
        _lib.check(self._lib.aeo_set_field_f32(self._h, FIELDS[name], a.ctypes.data_as(C.c_void_p)), self._h)

    def get_field_f32(self, name: str, out: Optional[np.ndarray] = None) -> np.ndarray:
        """get_field into an FP32 host array."""
        if out is None:
            out = np.empty(self.grid.storage_shape, dtype=np.float32)
        if out.dtype != np.float32 or out.shape != self.grid.storage_shape or not out.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous float32 array of the storage shape")
        _lib.check(self._lib.aeo_get_field_f32(self._h, FIELDS[name], out.ctypes.data_as(C.c_void_p)), self._h)
        return out

    def set_state(self, u, v, w, theta):
        self.set_field("u", u)
        self.set_field("v", v)
        self.set_field("w", w)
        self.set_field("theta", theta)

    def get_state(self):
        return tuple(self.get_field(n) for n in ("u", "v", "w", "theta"))

    def fill_uniform(self, name: str, seed: int, stream: int, amp: float, add: bool = False):
        _lib.check(self._lib.aeo_fill_uniform(self._h, FIELDS[name], seed, stream, amp, 1 if add else 0), self._h)

    # ---- stepping ---------------------------------------------------------------
    def step_rk3(self, dt: float, nsteps: int = 1):
        _lib.check(self._lib.aeo_step_rk3(self._h, float(dt), int(nsteps)), self._h)

    def step_rk3_async(self, dt: float, nsteps: int = 1):
        _lib.check(self._lib.aeo_step_rk3_async(self._h, float(dt), int(nsteps)), self._h)

    def synchronize(self):
        _lib.check(self._lib.aeo_synchronize(self._h), self._h)

    def step(self, dt: float, nsteps: int = 1):
        _lib.check(self._lib.aeo_step_euler(self._h, float(dt), int(nsteps)), self._h)

    def project(self):
        """One Chorin projection of the current velocity (dt = 1)."""
        _lib.check(self._lib.aeo_project(self._h), self._h)

    def init_isotropic(self, u_rms: float = 1.0, k_peak: float = 4.0, seed: int = 1, kmax: float = 0.0,
                       project: bool = True, target_rms: float = 0.0):
        """`isotropic_turbulence_field!` with the Passot-Pouquet spectrum
        (src/operators/spectra.jl:248-343) generated on the device; then an
        optional projection and rescaling to a per-component rms."""
        _lib.check(self._lib.aeo_init_isotropic(self._h, float(u_rms), float(k_peak), int(seed), float(kmax),
                                                1 if project else 0, float(target_rms)), self._h)

    def step_adaptive(self, constraints: "CFLConstraints" = None, nsteps: int = 1, dt_prev=None) -> dict:
        """`step_adaptive!` (src/TimeIntegration.jl:808-938) nsteps times: the
        CFL pick, the RK3 step and the guard run on the device; a failed guard
        retries the step from its unchanged start with half the dt.  Returns
        the stats of the last step (dt, limiter, ...) and the time advanced."""
        c = (constraints or CFLConstraints()).to_c()
        d = C.c_double(float(dt_prev) if dt_prev else 0.0)
        st = _lib.AeoAdaptiveStats()
        _lib.check(self._lib.aeo_step_adaptive(self._h, C.byref(c), int(nsteps), C.byref(d), C.byref(st)), self._h)
        return _stats(st)

    def cfl_diagnostics(self, constraints: "CFLConstraints" = None, dt_prev=None) -> dict:
        """`cfl_diagnostics` + `adaptive_dt` of the current state."""
        c = (constraints or CFLConstraints()).to_c()
        st = _lib.AeoAdaptiveStats()
        _lib.check(self._lib.aeo_cfl_diagnostics(self._h, C.byref(c), float(dt_prev or 0.0), C.byref(st)), self._h)
        return _stats(st)

    # ---- solver seam and diagnostics ------------------------------------------
    def pressure_solve(self, src: np.ndarray) -> np.ndarray:
        g = self.grid
        s = np.ascontiguousarray(src, dtype=np.float64)
        if s.shape != (g.nz, g.ny, g.nx):
            raise ValueError(f"source must have the interior shape {(g.nz, g.ny, g.nx)}")
        out = np.empty_like(s)
        _lib.check(self._lib.aeo_pressure_solve(self._h, _ptr(s), _ptr(out)), self._h)
        return out

    # ---- the implicit IBM correction ------------------------------------------------
    def set_ibm(self, mask=None, tau: float = 0.0):
        """implicit_ibm_correction! after every predictor (src/IBM.jl:295-300):
        a storage-shaped solid mask (None switches it off) and tau (0: the
        faces of solid cells are zeroed)."""
        if mask is None:
            _lib.check(self._lib.aeo_set_ibm(self._h, None, float(tau)), self._h)
            return
        m = np.ascontiguousarray(mask, dtype=np.uint8)
        if m.shape != self.grid.storage_shape:
            raise ValueError(f"mask must have the storage shape {self.grid.storage_shape}")
        _lib.check(self._lib.aeo_set_ibm(self._h, m.ctypes.data_as(C.c_void_p), float(tau)), self._h)

    # ---- positivity-preserving scalar advection -----------------------------------
    def advect_positive(self, u, v, w, phi, dt: float, scheme: str = "weno_z5", tend=None,
                        accumulate: bool = True) -> np.ndarray:
        """advect_positive! (src/AdvectionSchemes.jl:1141-1160): tend (a copy;
        zeros when None) with -div(u phi) added (accumulate) or written, the
        face fluxes limited so that phi + dt*tend stays non-negative under the
        first-order CFL condition.  Storage arrays with filled halos (>= 3)."""
        g = self.grid
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (u, v, w, phi)]
        for a in arrs:
            if a.shape != g.storage_shape:
                raise ValueError(f"arrays must have the storage shape {g.storage_shape}")
        if scheme not in ("weno_js5", "weno_z5"):
            raise ValueError("scheme must be weno_js5 or weno_z5")
        out = np.zeros(g.storage_shape) if tend is None else np.array(tend, dtype=np.float64, copy=True)
        if out.shape != g.storage_shape:
            raise ValueError(f"tend must have the storage shape {g.storage_shape}")
        _lib.check(self._lib.aeo_advect_positive(self._h, *[_ptr(a) for a in arrs], _ptr(out), float(dt),
                                                 ADVECTION[scheme], int(bool(accumulate))), self._h)
        return out

    def advect_positive_device(self, u, v, w, phi, tend, dt: float, scheme: str = "weno_z5",
                               accumulate: bool = True):
        """The same on device arrays (integer addresses, or objects with a
        data_ptr() such as torch tensors) of the working precision in the
        storage layout, enqueued on the domain's stream."""
        def addr(a):
            return C.c_void_p(a.data_ptr() if hasattr(a, "data_ptr") else int(a))
        _lib.check(self._lib.aeo_advect_positive_device(self._h, addr(u), addr(v), addr(w), addr(phi), addr(tend),
                                                        float(dt), ADVECTION[scheme], int(bool(accumulate))),
                   self._h)

    # ---- the PCG pressure solver (solver="pcg") --------------------------------
    def set_pcg(self, apertures=None, tol: float = 1e-8, maxit: int = 200):
        """The cut-cell face apertures (ax, ay, az) of shapes (nz, ny, nx+1),
        (nz, ny+1, nx), (nz+1, ny, nx) in [0, 1] (None: every face open) and
        the CG tolerance / iteration cap of every projection's solve."""
        g = self.grid
        if apertures is None:
            _lib.check(self._lib.aeo_set_pcg(self._h, None, None, None, float(tol), int(maxit)), self._h)
            return
        ax, ay, az = (np.ascontiguousarray(a, dtype=np.float64) for a in apertures)
        if ax.shape != (g.nz, g.ny, g.nx + 1) or ay.shape != (g.nz, g.ny + 1, g.nx) or az.shape != (g.nz + 1, g.ny, g.nx):
            raise ValueError("apertures must be (nz, ny, nx+1), (nz, ny+1, nx), (nz+1, ny, nx)")
        self._apertures = (ax, ay, az)
        _lib.check(self._lib.aeo_set_pcg(self._h, _ptr(ax), _ptr(ay), _ptr(az), float(tol), int(maxit)), self._h)

    def pcg_stats(self) -> dict:
        """The last projection's solve: iterations, status, ||r||, ||b||."""
        it, stt = C.c_int32(), C.c_int32()
        r, b = C.c_double(), C.c_double()
        _lib.check(self._lib.aeo_pcg_stats(self._h, C.byref(it), C.byref(stt), C.byref(r), C.byref(b)), self._h)
        from .multigrid import STATUS
        return {"iterations": it.value, "status": STATUS.get(stt.value, stt.value), "residual": r.value,
                "bnorm": b.value, "relative_residual": r.value / b.value if b.value > 0 else 0.0}

    def set_learned(self, net=None, stagnation: float = 0.9):
        """The learned U-Net preconditioner of every projection's solve (None:
        back to the multigrid cycle); kept alive by this object."""
        self._net = net
        _lib.check(self._lib.aeo_pcg_set_learned(self._h, net.handle if net is not None else None, float(stagnation)),
                   self._h)

    def set_open_boundaries(self, obc=None):
        """Open lateral faces from an OpenBoundarySet
        (open_boundary.open_boundary_conditions) on this domain's grid; None
        closes them again (periodic x and y)."""
        if obc is None:
            _lib.check(self._lib.aeo_set_open(self._h, 0, 0, None, None, None), self._h)
            self._open = None
            return
        if obc.grid.size != self.grid.size or obc.grid.halo != self.grid.halo:
            raise ValueError("the open boundaries were built for another grid")
        xp, yp, modes = obc.packed()
        _lib.check(self._lib.aeo_set_open(self._h, int(obc.open_x), int(obc.open_y), _ptr(xp), _ptr(yp),
                                          modes.ctypes.data_as(C.POINTER(C.c_int32))), self._h)
        rad = np.ascontiguousarray(obc.radiating, dtype=np.int32)
        xd, yd, _ = obc.packed(raw=True)
        xw, yw = obc.face_weights()
        _lib.check(self._lib.aeo_set_open_outflow(self._h, rad.ctypes.data_as(C.POINTER(C.c_int32)),
                                                  int(obc.correction_code), _ptr(xd), _ptr(yd), _ptr(xw), _ptr(yw)),
                   self._h)
        self._open = obc

    def open_planes(self):
        """The current plane buffers (x, y) in OpenBoundarySet.packed's layout."""
        xp, yp, _ = self._open.packed()
        _lib.check(self._lib.aeo_get_open_planes(self._h, _ptr(xp), _ptr(yp)), self._h)
        return xp, yp

    def open_checkpoint(self):
        """The state of the open faces a restart needs (open_boundary_checkpoint,
        src/boundary_conditions/open_boundary.jl:1282-1305): the plane buffers
        and, on a radiating set, the Orlanski history; None without open faces."""
        if getattr(self, "_open", None) is None:
            return None
        xp, yp = self.open_planes()
        out = {"planes_x": xp, "planes_y": yp}
        if self._open.radiating.any():
            g = self.grid
            NZ, NY, NX = g.storage_shape
            hx, hy, sc = np.zeros((4, 2, NZ, NY)), np.zeros((4, 2, NZ, NX)), np.zeros(2)
            _lib.check(self._lib.aeo_get_open_history(self._h, _ptr(hx), _ptr(hy), _ptr(sc)), self._h)
            out.update({"hist_x": hx, "hist_y": hy, "hist_set": float(sc[0]), "last_dt": float(sc[1])})
        return out

    def restore_open_checkpoint(self, state):
        """Copy an open_checkpoint back (restore_open_boundary_checkpoint!,
        :1307-1350): the faces must be built as the checkpointed ones."""
        if state is None:
            return
        if getattr(self, "_open", None) is None:
            raise ValueError("restore: the checkpoint has open faces, the domain none")
        xp, yp, _ = self._open.packed()
        if state["planes_x"].shape != xp.shape or state["planes_y"].shape != yp.shape:
            raise ValueError("restore: the open faces are built differently from the checkpoint's")
        if ("hist_x" in state) != bool(self._open.radiating.any()):
            raise ValueError("restore: the radiating faces differ from the checkpoint's")
        _lib.check(self._lib.aeo_set_open_planes(self._h, _ptr(np.ascontiguousarray(state["planes_x"])),
                                                 _ptr(np.ascontiguousarray(state["planes_y"]))), self._h)
        if "hist_x" in state:
            sc = np.array([state["hist_set"], state["last_dt"]])
            _lib.check(self._lib.aeo_set_open_history(self._h, _ptr(np.ascontiguousarray(state["hist_x"])),
                                                      _ptr(np.ascontiguousarray(state["hist_y"])), _ptr(sc)),
                       self._h)

    def open_ledger(self) -> dict:
        """Q, residual and delta of the last mass-flux correction on the device
        (a radiating open set)."""
        out = np.zeros(3)
        _lib.check(self._lib.aeo_open_ledger(self._h, _ptr(out)), self._h)
        return {"Q": out[0], "residual": out[1], "delta": out[2]}

    def pcg_harvest(self, cap: int = 10):
        """Residual -> error pairs from the run's own snapshot: the right-hand
        side b of the last projection's solve, solved again from zero by the
        plain MG-preconditioned CG.  Returns (b, x, [(r_k, x - x_k)]) as
        interior (nz, ny, nx) FP64 arrays, A (x - x_k) = r_k."""
        g = self.grid
        shape = (g.nz, g.ny, g.nx)
        b, x = np.empty(shape), np.empty(shape)
        rh, xh = np.empty((cap,) + shape), np.empty((cap,) + shape)
        cnt = C.c_int32()
        _lib.check(self._lib.aeo_pcg_harvest(self._h, int(cap), _ptr(b), _ptr(x), _ptr(rh), _ptr(xh), C.byref(cnt)),
                   self._h)
        return b, x, [(rh[k], x - xh[k]) for k in range(cnt.value)]

    def kinetic_energy(self) -> float:
        v = C.c_double()
        _lib.check(self._lib.aeo_kinetic_energy(self._h, C.byref(v)), self._h)
        return v.value

    def max_divergence(self) -> float:
        v = C.c_double()
        _lib.check(self._lib.aeo_max_divergence(self._h, C.byref(v)), self._h)
        return v.value

    def profile_step(self, dt: float) -> dict:
        """One RK3 step launch by launch with CUDA events between kernel
        groups: device milliseconds per kernel class (advances the state)."""
        n = len(_lib.KERNEL_CLASSES)
        buf = (C.c_double * n)()
        _lib.check(self._lib.aeo_profile_step(self._h, float(dt), buf, n), self._h)
        return {k: buf[i] for i, k in enumerate(_lib.KERNEL_CLASSES)}

    def launches_per_step(self) -> int:
        v = C.c_int32()
        _lib.check(self._lib.aeo_launches_per_step(self._h, C.byref(v)), self._h)
        return v.value

    @property
    def stream(self) -> int:
        return self._lib.aeo_stream(self._h)


def boussinesq_simulation(grid: Grid, *, nu=0.0, theta0=0.0, g=9.81, f_coriolis=0.0, c_s=0.0, pr_t=1 / 3,
                          flux_bot=0.0, flux_top=0.0, sponge_alpha=0.0, sponge_zstart=None,
                          advection="centred", precision="fp64", solver=None, device=0) -> Simulation:
    """`BoussinesqSimulation(mesh; ν, θ₀, g_accel, f_coriolis, C_s, Pr_t,
    θ_flux_bottom, θ_flux_top, sponge_α_max, sponge_z_start)`
    (src/Simulations.jl:232-246) on the B200."""
    spec = CoreSpec(grid=grid, core="boussinesq", advection=advection, solver=solver, precision=precision,
                    nu=nu, theta0=theta0, g=g, f_coriolis=f_coriolis, c_s=c_s, pr_t=pr_t, flux_bot=flux_bot,
                    flux_top=flux_top, sponge_alpha=sponge_alpha, sponge_zstart=sponge_zstart)
    return Simulation(spec, device)


def anelastic_spec(grid: Grid, rho_c, theta_c, **kw) -> CoreSpec:
    prof = anelastic_profiles(grid, rho_c, theta_c)
    return CoreSpec(grid=grid, core="anelastic", wc=prof["wc"], wf=prof["wf"], thf=prof["thf"], **kw)


def anelastic_simulation(grid: Grid, rho_c, theta_c, *, nu=0.0, g=9.81, f_coriolis=0.0, c_s=0.0, pr_t=1 / 3,
                         flux_bot=0.0, flux_top=0.0, sponge_alpha=0.0, sponge_zstart=None, precision="fp64",
                         device=0) -> Simulation:
    """The anelastic (W = rho_bar) sound-proof core (src/Anelastic.jl:1559,
    :1791-1948) with the direct FFT-tridiagonal weighted solver
    (DirectWeightedPoissonSolver, src/Anelastic.jl:987-1021)."""
    spec = anelastic_spec(grid, rho_c, theta_c, nu=nu, g=g, f_coriolis=f_coriolis, c_s=c_s, pr_t=pr_t,
                          flux_bot=flux_bot, flux_top=flux_top, sponge_alpha=sponge_alpha,
                          sponge_zstart=sponge_zstart, precision=precision)
    return Simulation(spec, device)


# reference-named free functions
def step_rk3(sim: Simulation, dt: float, nsteps: int = 1):
    sim.step_rk3(dt, nsteps)
    return sim


def step(sim: Simulation, dt: float, nsteps: int = 1):
    sim.step(dt, nsteps)
    return sim


def kinetic_energy(sim: Simulation) -> float:
    return sim.kinetic_energy()


def max_divergence(sim: Simulation) -> float:
    return sim.max_divergence()
