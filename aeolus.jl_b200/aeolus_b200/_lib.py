"""ctypes binding of libaeolus_b200.so (the C-ABI of include/aeolus_b200.h).

The library is built in-tree (aeolus_b200/lib/libaeolus_b200.so, see
`aeolus_b200.build`).  There is no fallback: if the library is missing or
a symbol is absent, loading raises.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libaeolus_b200.so")

# every entry point include/aeolus_b200.h and include/aeolus_b200_mgpcg.h declare
SYMBOLS = (
    "aeo_create", "aeo_destroy", "aeo_set_field", "aeo_get_field", "aeo_step_rk3", "aeo_step_euler",
    "aeo_pressure_solve", "aeo_project", "aeo_kinetic_energy", "aeo_max_divergence", "aeo_step_rk3_async",
    "aeo_synchronize", "aeo_profile_step", "aeo_launches_per_step", "aeo_stream", "aeo_fill_uniform",
    "aeo_pressure_solve_column_noalloc", "aeo_step_adaptive", "aeo_cfl_diagnostics", "aeo_init_isotropic", "aeo_last_error",
    "aeo_set_pcg", "aeo_pcg_stats", "aeo_pcg_set_learned", "aeo_pcg_harvest", "aeo_set_open", "aeo_set_open_outflow", "aeo_open_ledger", "aeo_get_open_planes", "aeo_set_open_planes", "aeo_get_open_history", "aeo_set_open_history", "aeo_advect_positive", "aeo_advect_positive_device", "aeo_set_ibm", "aeo_set_sgs_buoyancy", "aeo_set_lagrangian", "aeo_set_tke", "aeo_get_sgs_state", "aeo_set_sgs_state", "aeo_set_field_f32", "aeo_get_field_f32",
    "aeo_version",
    "aeo_mg_create", "aeo_mg_destroy", "aeo_mg_levels", "aeo_mg_solve", "aeo_mg_solve_device",
    "aeo_mg_vcycle_solve", "aeo_mg_apply", "aeo_mg_precondition", "aeo_mg_profile",
    "aeo_mg_launches_per_iteration", "aeo_mg_last_error", "aeo_mg_set_learned", "aeo_mg_solve_harvest",
    "aeo_unet_param_count", "aeo_unet_create", "aeo_unet_destroy", "aeo_unet_set_params", "aeo_unet_get_params",
    "aeo_unet_set_mask", "aeo_unet_set_out_scale", "aeo_unet_apply", "aeo_unet_gradients", "aeo_unet_train_step",
    "aeo_unet_activation", "aeo_unet_profile", "aeo_unet_last_error",
    "aeo_ghost_create", "aeo_ghost_destroy", "aeo_ghost_reconstruct", "aeo_ghost_reconstruct_host",
    "aeo_ghost_wall_stress", "aeo_ghost_wall_stress_host", "aeo_ghost_last_error",
)


class AeoConfig(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("hx", C.c_int32), ("hy", C.c_int32), ("hz", C.c_int32),
        ("lx", C.c_double), ("ly", C.c_double), ("lz", C.c_double),
        ("x0", C.c_double), ("y0", C.c_double), ("z0", C.c_double),
        ("bc_x", C.c_int32), ("bc_y", C.c_int32), ("bc_z", C.c_int32),
        ("stretched", C.c_int32), ("core", C.c_int32), ("advection", C.c_int32),
        ("solver", C.c_int32), ("precision", C.c_int32),
        ("nu", C.c_double), ("theta0", C.c_double), ("g", C.c_double), ("f_coriolis", C.c_double),
        ("c_s", C.c_double), ("pr_t", C.c_double), ("flux_bot", C.c_double), ("flux_top", C.c_double),
        ("sponge_alpha", C.c_double), ("sponge_zstart", C.c_double),
        ("device", C.c_int32), ("sgs_model", C.c_int32),
    ]


class AeoCfl(C.Structure):
    """CFLConstraints + the guard limits of step_adaptive! (src/TimeIntegration.jl:127-153, :823-835)."""
    _fields_ = [
        ("c_advective", C.c_double), ("c_diffusive", C.c_double), ("c_buoyancy", C.c_double),
        ("c_coriolis", C.c_double), ("dt_min", C.c_double), ("dt_max", C.c_double), ("growth_max", C.c_double),
        ("divergence_tol", C.c_double), ("max_velocity", C.c_double), ("max_retries", C.c_int32),
    ]


class AeoAdaptiveStats(C.Structure):
    _fields_ = [
        ("dt", C.c_double), ("t_advanced", C.c_double), ("limiter", C.c_int32), ("retries", C.c_int32),
        ("advective_rate", C.c_double), ("nut_max", C.c_double), ("brunt_vaisala", C.c_double),
        ("max_divergence", C.c_double), ("max_speed", C.c_double),
    ]


class AeoMgConfig(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
        ("bc_x", C.c_int32), ("bc_y", C.c_int32), ("bc_z", C.c_int32),
        ("precision", C.c_int32), ("precond", C.c_int32), ("flexible", C.c_int32),
        ("tol", C.c_double), ("maxit", C.c_int32), ("nu1", C.c_int32), ("nu2", C.c_int32),
        ("coarse_sweeps", C.c_int32), ("min_size", C.c_int32), ("device", C.c_int32),
    ]


class AeoMgStats(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("status", C.c_int32), ("residual", C.c_double),
                ("bnorm", C.c_double), ("curvature", C.c_double), ("fallback_at", C.c_int32)]


LIMITERS = ("advective", "diffusive", "buoyancy", "coriolis", "sgs", "growth", "dt_min", "dt_max", "retried")

_lib = None

KERNEL_CLASSES = ("sgs", "sweep", "div_fftx", "ffty", "zsolve", "ifftx", "correct", "halo")

STATUS = {0: "ok", 1: "argument", 2: "cuda", 3: "numerical", 4: "state"}


class AeolusError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"aeolus_b200 [{STATUS.get(status, status)}]: {msg}")
        self.status = status


class NumericalFailure(AeolusError):
    """Non-finite state or failed solve (the reference's NumericalFailure,
    src/TimeIntegration.jl:610)."""


def load():
    """Load the shared library (raises when it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libaeolus_b200.so not built: {LIB_PATH} is missing (run aeolus_b200.build())")
    lib = C.CDLL(LIB_PATH)
    for s in SYMBOLS:
        if not hasattr(lib, s):
            raise ImportError(f"libaeolus_b200.so lacks the symbol {s}")
    P = C.c_void_p
    D = C.POINTER(C.c_double)
    lib.aeo_create.argtypes = [C.POINTER(AeoConfig), D, D, D, D, C.POINTER(P)]
    lib.aeo_destroy.argtypes = [P]
    lib.aeo_set_field.argtypes = [P, C.c_int32, D]
    lib.aeo_get_field.argtypes = [P, C.c_int32, D]
    lib.aeo_step_rk3.argtypes = [P, C.c_double, C.c_int32]
    lib.aeo_step_rk3_async.argtypes = [P, C.c_double, C.c_int32]
    lib.aeo_step_euler.argtypes = [P, C.c_double, C.c_int32]
    lib.aeo_synchronize.argtypes = [P]
    lib.aeo_pressure_solve.argtypes = [P, D, D]
    lib.aeo_project.argtypes = [P]
    lib.aeo_kinetic_energy.argtypes = [P, D]
    lib.aeo_max_divergence.argtypes = [P, D]
    I32 = C.POINTER(C.c_int32)
    lib.aeo_set_pcg.argtypes = [P, D, D, D, C.c_double, C.c_int32]
    lib.aeo_set_ibm.argtypes = [P, C.c_void_p, C.c_double]
    lib.aeo_set_sgs_buoyancy.argtypes = [P, C.c_void_p]
    lib.aeo_set_lagrangian.argtypes = [P, C.c_double, C.c_double, C.c_double]
    lib.aeo_set_tke.argtypes = [P, C.c_double, C.c_double, C.c_double, C.c_int32]
    lib.aeo_get_sgs_state.argtypes = [P, C.c_void_p]
    lib.aeo_set_sgs_state.argtypes = [P, C.c_void_p]
    lib.aeo_set_field_f32.argtypes = [P, C.c_int32, C.c_void_p]
    lib.aeo_get_field_f32.argtypes = [P, C.c_int32, C.c_void_p]
    lib.aeo_advect_positive.argtypes = [P, D, D, D, D, D, C.c_double, C.c_int32, C.c_int32]
    lib.aeo_advect_positive_device.argtypes = [P, P, P, P, P, P, C.c_double, C.c_int32, C.c_int32]
    lib.aeo_pcg_stats.argtypes = [P, I32, I32, D, D]
    lib.aeo_pcg_set_learned.argtypes = [P, P, C.c_double]
    lib.aeo_pcg_harvest.argtypes = [P, C.c_int32, D, D, D, D, I32]
    lib.aeo_set_open.argtypes = [P, C.c_int32, C.c_int32, D, D, I32]
    lib.aeo_set_open_outflow.argtypes = [P, I32, C.c_int32, D, D, D, D]
    lib.aeo_open_ledger.argtypes = [P, D]
    lib.aeo_get_open_planes.argtypes = [P, D, D]
    lib.aeo_set_open_planes.argtypes = [P, D, D]
    lib.aeo_get_open_history.argtypes = [P, D, D, D]
    lib.aeo_set_open_history.argtypes = [P, D, D, D]
    lib.aeo_profile_step.argtypes = [P, C.c_double, D, C.c_int32]
    lib.aeo_launches_per_step.argtypes = [P, C.POINTER(C.c_int32)]
    lib.aeo_stream.argtypes = [P]
    lib.aeo_stream.restype = C.c_void_p
    lib.aeo_fill_uniform.argtypes = [P, C.c_int32, C.c_uint64, C.c_uint32, C.c_double, C.c_int32]
    lib.aeo_pressure_solve_column_noalloc.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_double,
                                                      D, D, D, D, D, D, P, P, P]
    lib.aeo_step_adaptive.argtypes = [P, C.POINTER(AeoCfl), C.c_int32, D, C.POINTER(AeoAdaptiveStats)]
    lib.aeo_cfl_diagnostics.argtypes = [P, C.POINTER(AeoCfl), C.c_double, C.POINTER(AeoAdaptiveStats)]
    lib.aeo_init_isotropic.argtypes = [P, C.c_double, C.c_double, C.c_uint64, C.c_double, C.c_int32, C.c_double]
    lib.aeo_last_error.argtypes = [P]
    lib.aeo_last_error.restype = C.c_char_p
    lib.aeo_version.restype = C.c_char_p
    lib.aeo_mg_create.argtypes = [C.POINTER(AeoMgConfig), D, D, D, C.POINTER(P)]
    lib.aeo_mg_destroy.argtypes = [P]
    lib.aeo_mg_levels.argtypes = [P, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
    for f in (lib.aeo_mg_solve, lib.aeo_mg_vcycle_solve):
        f.argtypes = [P, D, D, C.POINTER(AeoMgStats)]
    lib.aeo_mg_solve_device.argtypes = [P, P, P, C.POINTER(AeoMgStats)]
    lib.aeo_mg_apply.argtypes = [P, D, D]
    lib.aeo_mg_precondition.argtypes = [P, D, D]
    lib.aeo_mg_profile.argtypes = [P, C.c_int32, C.c_int32, D]
    lib.aeo_mg_launches_per_iteration.argtypes = [P]
    lib.aeo_mg_last_error.argtypes = [P]
    lib.aeo_mg_last_error.restype = C.c_char_p
    lib.aeo_mg_set_learned.argtypes = [P, P, C.c_double]
    lib.aeo_mg_solve_harvest.argtypes = [P, D, D, C.POINTER(AeoMgStats), D, D, C.c_int32, C.POINTER(C.c_int32)]
    F = C.POINTER(C.c_float)
    lib.aeo_unet_param_count.restype = C.c_int64
    lib.aeo_unet_create.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_uint64, C.c_int32, C.POINTER(P)]
    lib.aeo_unet_destroy.argtypes = [P]
    lib.aeo_unet_set_params.argtypes = [P, F]
    lib.aeo_unet_get_params.argtypes = [P, F, F]
    lib.aeo_unet_set_mask.argtypes = [P, F]
    lib.aeo_unet_set_out_scale.argtypes = [P, C.c_double]
    lib.aeo_unet_apply.argtypes = [P, D, D]
    lib.aeo_unet_gradients.argtypes = [P, D, D, D]
    lib.aeo_unet_train_step.argtypes = [P, D, D, C.c_double, D]
    lib.aeo_unet_activation.argtypes = [P, C.c_int32, F]
    lib.aeo_unet_profile.argtypes = [P, C.c_int32, C.c_int32, D]
    lib.aeo_unet_last_error.argtypes = [P]
    lib.aeo_unet_last_error.restype = C.c_char_p
    I64 = C.POINTER(C.c_int64)
    lib.aeo_ghost_create.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_int64, I64, I64, D, D, D, D,
                                     C.POINTER(C.c_uint8), C.c_int32, C.POINTER(P)]
    lib.aeo_ghost_destroy.argtypes = [P]
    lib.aeo_ghost_reconstruct.argtypes = [P, P, C.c_int32, C.c_int32, C.c_double, C.c_double, P]
    lib.aeo_ghost_reconstruct_host.argtypes = [P, D, C.c_int32, C.c_double, C.c_double]
    lib.aeo_ghost_wall_stress.argtypes = [P, P, P, P, P, P, P, C.c_int32, D, C.c_double, C.c_double, P, P, P]
    lib.aeo_ghost_wall_stress_host.argtypes = [P, D, D, D, D, D, D, C.c_int32, D, C.c_double, C.c_double, D, D]
    lib.aeo_ghost_last_error.argtypes = [P]
    lib.aeo_ghost_last_error.restype = C.c_char_p
    for s in SYMBOLS:
        f = getattr(lib, s)
        if s not in ("aeo_stream", "aeo_last_error", "aeo_version", "aeo_mg_last_error", "aeo_unet_last_error",
                     "aeo_unet_param_count", "aeo_ghost_last_error"):
            f.restype = C.c_int32
    _lib = lib
    return lib


def check(status: int, handle=None, mg=False, unet=False, ghost=False):
    if status == 0:
        return
    lib = load()
    f = (lib.aeo_ghost_last_error if ghost else lib.aeo_unet_last_error if unet else
         (lib.aeo_mg_last_error if mg else lib.aeo_last_error))
    msg = f(handle).decode(errors="replace")
    if status == 3:
        raise NumericalFailure(status, msg)
    if status == 1:
        raise ValueError(f"aeolus_b200: {msg}")
    raise AeolusError(status, msg)
