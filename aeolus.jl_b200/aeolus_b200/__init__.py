"""aeolus_b200 -- the B200 (sm_100a) dynamical-core step of Aeolus.jl.

Host-side Python mirror of the reference's step-core interface over the
C-ABI library libaeolus_b200.so (include/aeolus_b200.h).  The CUDA path is
the only path: importing the simulation classes loads the library and raises
if it has not been built.
"""
import os
import subprocess

from .grids import (PERIODIC, WALL, Grid, regular_grid, stretched_grid, stretching_ratio, tanh_beta_for_first_cell,
                    tanh_faces)
from .reference_state import anelastic_profiles, exponential_density
from .spec import CoreSpec

_PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def build(verbose: bool = False) -> str:
    """Compile libaeolus_b200.so for sm_100a in-tree (make) and return its path."""
    r = subprocess.run(["make", "-C", _PKG_ROOT], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"building libaeolus_b200.so failed:\n{r.stdout}\n{r.stderr}")
    if verbose:
        print(r.stdout)
    from ._lib import LIB_PATH
    return LIB_PATH


def __getattr__(name):
    # the ctypes-backed classes load the library on first use
    if name in ("Simulation", "boussinesq_simulation", "anelastic_simulation", "anelastic_spec", "step_rk3",
                "step", "kinetic_energy", "max_divergence"):
        from . import simulation
        return getattr(simulation, name)
    raise AttributeError(name)
