"""The description of one domain's dynamical core: grid + physics + solver.

`CoreSpec` carries what the reference spreads over the constructor keywords
of `BoussinesqSimulation` (src/Simulations.jl:232-246), the sound-proof
simulation (src/Anelastic.jl:1559) and the TOML `[core]` / `[advection]` /
`[sgs]` / pressure-solver sections (src/config/simulation_driver.jl:416-495).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from .grids import PERIODIC, WALL, Grid

CORES = {"boussinesq": 0, "anelastic": 1}
ADVECTION = {"centred": 0, "weno_js5": 1, "weno_z5": 2}
SGS_MODELS = {"smagorinsky": 0, "vreman": 1, "sigma": 2, "amd": 3, "dynamic": 4, "lagrangian": 6, "tke": 7}
SOLVERS = {"fft": 0, "column": 1, "pcg": 2}
PRECISIONS = {"fp64": 0, "fp32_mixed": 1}
FIELDS = {"u": 0, "v": 1, "w": 2, "theta": 3, "p": 4, "nut": 5}


@dataclass
class CoreSpec:
    grid: Grid
    core: str = "boussinesq"
    advection: str = "centred"
    solver: Optional[str] = None        # default: fft when z is periodic, else column
    precision: str = "fp64"
    nu: float = 0.0
    theta0: float = 0.0
    g: float = 9.81
    f_coriolis: float = 0.0
    c_s: float = 0.0
    sgs: str = "smagorinsky"            # the closure when c_s > 0: smagorinsky, vreman (c = 2.5 c_s^2),
                                        # sigma (c_s is C_sigma, 1.35 in the reference) or amd (c_s is the
                                        # AMD constant C, 0.3 in the reference; its own kappa_t) or dynamic
                                        # (Germano-Lilly, plane-averaged; c_s is the clip cs_max, 0.5)
    averaging: str = "plane"            # the dynamic closure's <.>: "plane" (each level) or "local" (each
                                        # cell its own clipped ratio; DynamicSmagorinsky(averaging = :local))
    # sgs = "lagrangian" (LagrangianDynamicSmagorinsky; c_s is the clip cs_max, 0.5): the initial
    # coefficient C0, the time-scale factor theta and a fixed memory_time (None: MLC96's T)
    lag_c0: float = 0.16
    lag_theta: float = 1.5
    lag_memory_time: Optional[float] = None
    # sgs = "tke" (TKEClosure, Deardorff 1980 / Moeng 1984; c_s is c_k, 0.1): c_eps0, c_eps1, c_l, the
    # dissipation form ("semi_implicit" or "exact") and a uniform initial e (m^2 s^-2)
    tke_c_eps0: float = 0.19
    tke_c_eps1: float = 0.51
    tke_c_l: float = 0.76
    tke_dissipation: str = "semi_implicit"
    tke_e0: float = 0.0
    pr_t: float = 1.0 / 3.0
    flux_bot: float = 0.0
    flux_top: float = 0.0
    sponge_alpha: float = 0.0
    sponge_zstart: Optional[float] = None
    wc: Optional[np.ndarray] = field(default=None, repr=False)
    wf: Optional[np.ndarray] = field(default=None, repr=False)
    thf: Optional[np.ndarray] = field(default=None, repr=False)
    thc: Optional[np.ndarray] = field(default=None, repr=False)   # theta_bar at the Nz cell centres (the
                                        # AMD closure's buoyancy g/theta_bar(z) on the sound-proof core)

    def __post_init__(self):
        if self.core not in CORES:
            raise ValueError(f"core must be one of {list(CORES)}, got {self.core!r}")
        if self.advection not in ADVECTION:
            raise ValueError(f"advection must be one of {list(ADVECTION)}, got {self.advection!r}")
        if self.precision not in PRECISIONS:
            raise ValueError(f"precision must be one of {list(PRECISIONS)}, got {self.precision!r}")
        if self.solver is None:
            # _default_solver, src/Simulations.jl:1137-1144
            self.solver = "fft" if self.grid.bc_z == PERIODIC else "column"
        if self.solver not in SOLVERS:
            raise ValueError(f"solver must be one of {list(SOLVERS)}, got {self.solver!r}")
        if self.sponge_zstart is None:
            self.sponge_zstart = self.grid.origin[2] + self.grid.extent[2]
        if self.core == "anelastic":
            if self.wc is None or self.wf is None:
                raise ValueError("the anelastic core needs the padded weights wc and wf")
            if self.grid.bc_z != WALL:
                raise ValueError("the anelastic core needs walls in z")
            nzs = self.grid.nz + 2 * self.grid.halo[2]
            self.wc = np.ascontiguousarray(self.wc, dtype=np.float64)
            self.wf = np.ascontiguousarray(self.wf, dtype=np.float64)
            if self.wc.shape != (nzs,) or self.wf.shape != (nzs + 1,):
                raise ValueError(f"wc needs {nzs} and wf {nzs + 1} storage levels")
            if self.thf is not None:
                self.thf = np.ascontiguousarray(self.thf, dtype=np.float64)
                if self.thf.shape != (nzs + 1,):
                    raise ValueError(f"thf needs {nzs + 1} storage levels")
        if self.advection != "centred":
            if self.grid.stretched or self.core != "boussinesq":
                raise ValueError("WENO advection is defined on a uniform Boussinesq grid "
                                 "(momentum_advect_weno_z!, src/AdvectionSchemes.jl:1195)")
            if min(self.grid.halo) < 3:
                raise ValueError("WENO-5 needs halo >= 3 in every direction")
        if self.c_s != 0 and not self.pr_t > 0:
            raise ValueError("pr_t must be positive")
        if self.sgs not in SGS_MODELS:
            raise ValueError(f"sgs must be one of {list(SGS_MODELS)}, got {self.sgs!r}")
        if self.averaging not in ("plane", "local"):
            raise ValueError(f"averaging must be 'plane' or 'local', got {self.averaging!r} (src/Operators.jl:558-559)")
        if self.sgs in ("vreman", "sigma", "amd", "dynamic", "lagrangian", "tke") and self.grid.stretched:
            raise ValueError("the Vreman, sigma and AMD closures take a RegularGrid only (compute_vreman_nut!, "
                             "src/operators/sgs_amd_vreman.jl:280-284; compute_amd_coefficients!, :102-107; "
                             "compute_sigma_nut!, src/operators/sigma_closure.jl:208-212)")
        if self.sgs in ("dynamic", "lagrangian") and self.c_s != 0 and min(self.grid.halo) < 2:
            raise ValueError("the dynamic Smagorinsky closures need halos of at least 2 (src/Operators.jl:556-557, "
                             "src/operators/lagrangian_sgs.jl:170-171)")
        if self.sgs == "tke" and self.c_s != 0:
            if self.core != "boussinesq" or min(self.grid.halo) < 3:
                raise ValueError("the TKE closure runs on the Boussinesq core (theta0 its buoyancy reference) with "
                                 "halos >= 3 (the WENO-Z5 transport of e, src/PrognosticSGS.jl:354-356)")
            if self.tke_dissipation not in ("semi_implicit", "exact"):
                raise ValueError(f"dissipation must be 'semi_implicit' or 'exact', got {self.tke_dissipation!r} "
                                 "(src/PrognosticSGS.jl:332-333)")
            if not (self.tke_c_eps0 >= 0 and self.tke_c_eps1 >= 0 and self.tke_c_l > 0 and self.tke_e0 >= 0):
                raise ValueError("c_eps0, c_eps1 >= 0, c_l > 0 and e0 >= 0 required")
        if self.sgs == "lagrangian":
            if not (self.lag_c0 > 0 and self.lag_theta > 0):
                raise ValueError("lag_c0 and lag_theta must be positive")
            if self.lag_memory_time is not None and not self.lag_memory_time > 0:
                raise ValueError(f"memory_time must be positive (or None for MLC96's T), got {self.lag_memory_time} "
                                 "(src/operators/lagrangian_sgs.jl:172-173)")
        if self.sgs == "amd" and self.c_s != 0 and self.core == "anelastic":
            if self.thc is None:
                raise ValueError("the AMD closure on the sound-proof core needs thc, theta_bar at the cell centres "
                                 "(its buoyancy parameter g/theta_bar(z_k), src/operators/sgs_amd_vreman.jl:331-345)")
            self.thc = np.ascontiguousarray(self.thc, dtype=np.float64)
            if self.thc.shape != (self.grid.nz,) or np.any(self.thc <= 0):
                raise ValueError(f"thc needs {self.grid.nz} positive values")


def sgs_model_code(spec) -> int:
    """The C-ABI's AEO_SGS_* of a spec (the dynamic closure with :local
    averaging is its own code)."""
    if spec.sgs == "dynamic" and spec.averaging == "local":
        return 5
    return SGS_MODELS[spec.sgs]


def sgs_buoyancy_levels(spec):
    """The AMD closure's per-level buoyancy parameter g/theta_bar(z_k) of a
    sound-proof spec (None where the closure takes g/theta0 or is off)."""
    if spec.sgs == "amd" and spec.c_s != 0 and spec.core == "anelastic":
        return spec.g / spec.thc
    return None
