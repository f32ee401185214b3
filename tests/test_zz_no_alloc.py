"""The allocation-free column pressure solve against the handle's solve.

`aeo_pressure_solve_column_noalloc` serves callers that cannot call
cudaMalloc (a runtime whose device memory must come from its own pool, an
application that reserves all memory up front, a loop that cannot take
cudaMalloc's implicit synchronisation): every input and output is the
caller's device array and its scratch is a static array of the library.
Two calls in a row, with different sources, must each match
`aeo_pressure_solve` of a domain handle (same operator) to the tolerance of
the pressure-solve parity tests, so nothing of the first call's scratch
leaks into the second.  This file is collected last.
"""
import ctypes as C

import numpy as np
import pytest

from aeolus_b200 import CoreSpec, _lib, stretched_grid, tanh_faces

pytestmark = pytest.mark.gpu

_D = C.POINTER(C.c_double)


def column_coefficients(zf):
    """ColumnTridiagonalSolver(dzc, dzf) coefficients (src/PressureSolvers.jl:686-700)."""
    nz = len(zf) - 1
    dzc = np.diff(zf)
    zc = 0.5 * (zf[:-1] + zf[1:])
    dzf = np.empty(nz + 1)
    dzf[0] = dzc[0]
    dzf[1:nz] = zc[1:] - zc[:-1]
    dzf[nz] = dzc[-1]
    lower = np.zeros(nz)
    upper = np.zeros(nz)
    lower[1:] = 1 / (dzc[1:] * dzf[1:nz])
    upper[:-1] = 1 / (dzc[:-1] * dzf[1:nz])
    return lower, upper, np.ones(nz), dzc.copy(), dzf, dzc.copy()


def noalloc_solve(lib, g, coefs, src):
    import torch
    s = torch.from_numpy(np.ascontiguousarray(src)).cuda()
    p = torch.empty_like(s)
    torch.cuda.synchronize()
    arrs = [np.ascontiguousarray(c, dtype=np.float64) for c in coefs]
    st = lib.aeo_pressure_solve_column_noalloc(g.nx, g.ny, g.nz, g.extent[0], g.extent[1],
                                               *[a.ctypes.data_as(_D) for a in arrs],
                                               C.c_void_p(s.data_ptr()), C.c_void_p(p.data_ptr()), None)
    assert st == 0, lib.aeo_last_error(None)
    torch.cuda.synchronize()
    return p.cpu().numpy()


def _twice_against_the_handle(shape, extent, zf, seed):
    from aeolus_b200.simulation import Simulation
    lib = _lib.load()
    nx, ny, nz = shape
    g = stretched_grid(shape, extent, zf)
    sim = Simulation(CoreSpec(grid=g))  # FP64, walls in z: the column solver
    coefs = column_coefficients(zf)
    rng = np.random.default_rng(seed)
    for call in range(2):
        src = rng.standard_normal((nz, ny, nx)) * (1 + 10 * call)
        src -= src.mean()
        ref = sim.pressure_solve(src)
        out = noalloc_solve(lib, g, coefs, src)
        assert np.abs(out - ref).max() <= 1e-12 * np.abs(ref).max(), f"call {call + 1}"
    sim.close()


def test_noalloc_column_solve_matches_the_handle_solve_twice():
    nz = 24
    _twice_against_the_handle((64, 32, nz), (640.0, 320.0, 300.0), tanh_faces(nz, 300.0, 1.4), 11)


@pytest.mark.parametrize("shape", [(16, 16, 600), (16, 16, 800)])
def test_noalloc_deep_columns_match_the_handle_solve_twice(shape):
    """Columns deep enough that the column solve's shared memory exceeds the
    default 48 KiB (the launch raises the limit first)."""
    nz = shape[2]
    _twice_against_the_handle(shape, (10.0 * shape[0], 10.0 * shape[1], 3000.0), tanh_faces(nz, 3000.0, 1.2), 12)


def test_noalloc_refuses_a_capturing_stream_and_a_zero_measure():
    import torch
    lib = _lib.load()
    nz = 8
    zf = np.linspace(0.0, 80.0, nz + 1)
    arrs = [np.ascontiguousarray(c) for c in column_coefficients(zf)]
    s = torch.zeros((nz, 8, 8), dtype=torch.float64, device="cuda")
    p = torch.empty_like(s)
    ptrs = [a.ctypes.data_as(_D) for a in arrs]
    side = torch.cuda.Stream()
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=side):
        st = lib.aeo_pressure_solve_column_noalloc(8, 8, nz, 80.0, 80.0, *ptrs, C.c_void_p(s.data_ptr()),
                                                   C.c_void_p(p.data_ptr()), C.c_void_p(side.cuda_stream))
    assert st == 1
    assert b"capturing" in lib.aeo_last_error(None)
    zero = [a.copy() for a in arrs]
    zero[3][:] = 0.0   # measure
    st = lib.aeo_pressure_solve_column_noalloc(8, 8, nz, 80.0, 80.0, *[a.ctypes.data_as(_D) for a in zero],
                                               C.c_void_p(s.data_ptr()), C.c_void_p(p.data_ptr()), None)
    assert st == 1
    assert b"measure" in lib.aeo_last_error(None)


def test_noalloc_rejects_a_grid_beyond_its_scratch():
    lib = _lib.load()
    nz = 256
    zf = np.linspace(0.0, 1.0, nz + 1)
    arrs = [np.ascontiguousarray(c) for c in column_coefficients(zf)]
    st = lib.aeo_pressure_solve_column_noalloc(512, 512, nz, 1.0, 1.0, *[a.ctypes.data_as(_D) for a in arrs],
                                               None, None, None)
    assert st == 1
    st = lib.aeo_pressure_solve_column_noalloc(512, 512, nz, 1.0, 1.0, *[a.ctypes.data_as(_D) for a in arrs],
                                               C.c_void_p(16), C.c_void_p(16), None)
    assert st == 1
    assert b"32 MiB" in lib.aeo_last_error(None)
