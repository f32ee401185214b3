"""Host-side logic and the C-ABI library's symbol table (CPU only: no CUDA
call is made)."""
import ctypes as C
import glob
import os
import re

import numpy as np
import pytest

from aeolus_b200 import CoreSpec, regular_grid, stretched_grid, stretching_ratio, tanh_beta_for_first_cell, tanh_faces
from aeolus_b200 import _lib
from aeolus_b200.reference_state import anelastic_profiles, exponential_density, logmean, pad_center, pad_face

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b(aeo_[a-z0-9_]+)\s*\(", src):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(_lib.LIB_PATH)
    syms = declared_symbols()
    assert "aeo_create" in syms and "aeo_step_rk3" in syms
    for s in sorted(syms):
        assert hasattr(lib, s), f"libaeolus_b200.so does not export {s}"
    assert set(_lib.SYMBOLS) == syms


def test_library_loads_and_reports_version():
    lib = _lib.load()
    assert b"sm_100a" in lib.aeo_version()


def test_create_rejects_bad_config_without_touching_the_gpu():
    lib = _lib.load()
    cfg = _lib.AeoConfig()
    cfg.nx, cfg.ny, cfg.nz = 12, 16, 16      # nx not a power of two
    cfg.hx = cfg.hy = cfg.hz = 3
    cfg.lx = cfg.ly = cfg.lz = 1.0
    h = C.c_void_p()
    st = lib.aeo_create(C.byref(cfg), None, None, None, None, C.byref(h))
    assert st == 1 and not h.value
    assert b"powers of two" in lib.aeo_last_error(None)


def test_tanh_grid_of_the_convective_boundary_layer():
    # 2000 m over 128 levels, first cell 8 m, adjacent ratio <= 1.05
    beta = tanh_beta_for_first_cell(128, 2000.0, 8.0)
    zf = tanh_faces(128, 2000.0, beta)
    assert abs(np.diff(zf)[0] - 8.0) < 1e-9
    assert stretching_ratio(zf) <= 1.05
    assert zf[0] == 0.0 and zf[-1] == 2000.0
    assert 1.07 < beta < 1.08


def test_logmean_and_padding():
    assert logmean(2.0, 2.0) == 2.0
    assert abs(logmean(1.2, 1.1) - (0.1 / np.log(1.2 / 1.1))) < 1e-14
    assert abs(logmean(1.0, 1.0 + 1e-6) - (1.0 + 0.5e-6)) < 1e-12
    v = np.array([1.0, 0.9, 0.81])
    p = pad_center(v, 2)
    assert np.allclose(p, [1 / 0.81, 1 / 0.9, 1.0, 0.9, 0.81, 0.729, 0.6561])
    f = pad_face(np.array([1.0, 0.9, 0.81, 0.729]), 2, 3)
    assert len(f) == 3 + 4 + 1 and f[2] == 1.0 and f[5] == 0.729


def test_anelastic_profiles_wall_faces_mirror_the_cells():
    g = stretched_grid((8, 8, 10), (100.0, 100.0, 1000.0), tanh_faces(10, 1000.0, 1.5))
    rho = exponential_density(g)
    prof = anelastic_profiles(g, rho, np.full(10, 300.0))
    hz = g.halo[2]
    assert prof["wf"][hz] == rho[0] and prof["wf"][hz + 10] == rho[-1]
    assert np.all(prof["wf"][hz + 1:hz + 10] < np.maximum(rho[:-1], rho[1:]))
    assert np.all(prof["wc"][hz:hz + 10] == rho)
    assert np.allclose(prof["thf"][hz:hz + 11], 300.0)


def test_spec_validation():
    g = regular_grid((16, 16, 16), (1, 1, 1))
    with pytest.raises(ValueError):
        CoreSpec(grid=g, advection="weno_js5", core="anelastic")
    with pytest.raises(ValueError):
        CoreSpec(grid=regular_grid((16, 16, 16), (1, 1, 1), halo=(2, 2, 2)), advection="weno_z5")
    with pytest.raises(ValueError):
        CoreSpec(grid=g, core="anelastic")
    assert CoreSpec(grid=g).solver == "fft"
    assert CoreSpec(grid=regular_grid((16, 16, 16), (1, 1, 1), bc_z="wall")).solver == "column"


def test_pcg_solver_takes_any_core_and_column():
    """The cut-cell MG-PCG projection carries the density weights and the
    stretched metric in its operator, so every core and column accepts it;
    WENO advection stays on uniform Boussinesq grids."""
    from aeolus_b200 import CoreSpec, regular_grid, stretched_grid, tanh_faces
    from aeolus_b200.reference_state import anelastic_profiles, exponential_density
    g = regular_grid((32, 32, 16), (64.0, 64.0, 32.0), halo=(3, 3, 3), bc_z="wall")
    assert CoreSpec(grid=g, solver="pcg").solver == "pcg"
    gs = stretched_grid((32, 32, 16), (64.0, 64.0, 400.0), tanh_faces(16, 400.0, 1.5))
    assert CoreSpec(grid=gs, solver="pcg").solver == "pcg"
    prof = anelastic_profiles(gs, exponential_density(gs), 300.0 + 0 * gs.znodes("c"))
    assert CoreSpec(grid=gs, core="anelastic", solver="pcg", wc=prof["wc"], wf=prof["wf"]).solver == "pcg"
    with pytest.raises(ValueError):
        CoreSpec(grid=gs, solver="pcg", advection="weno_js5")
