"""Shared inputs of the positivity-preserving advection tests (the seeded
case of aeolus_b200.inputs.tracer_case on small grids)."""
from aeolus_b200 import CoreSpec, regular_grid
from aeolus_b200.inputs import tracer_case as case  # noqa: F401


def grid(n=(32, 16, 16), bc_z="periodic"):
    return regular_grid(n, (1.0, 0.5, 0.5), halo=(3, 3, 3), bc_z=bc_z)


def spec(g, precision="fp64"):
    return CoreSpec(grid=g, advection="weno_z5", precision=precision)
