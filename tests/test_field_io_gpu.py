"""Host field transfers in FP32 (aeo_set_field_f32 / aeo_get_field_f32): the
same storage layout and halo composite as the FP64 calls; on an FP32-mixed
domain a round trip returns the FP32 values exactly (theta too, whose
stored offset is applied on the way in and out), and the FP32 read of any
domain is the FP32 rounding of its FP64 read."""
import numpy as np
import pytest

from aeolus_b200 import CoreSpec, regular_grid

pytestmark = pytest.mark.gpu


def test_fp32_round_trip_and_consistency_with_fp64():
    from aeolus_b200.simulation import Simulation
    g = regular_grid((32, 16, 8), (1.0, 0.5, 0.25), halo=(3, 3, 3), bc_z="wall")
    rng = np.random.default_rng(3)
    for prec in ("fp32_mixed", "fp64"):
        s = Simulation(CoreSpec(grid=g, theta0=300.0, precision=prec))
        for name, base in (("u", 0.0), ("theta", 300.0)):
            a = (base + rng.standard_normal(g.storage_shape)).astype(np.float32)
            s.set_field_f32(name, a)
            b32 = s.get_field_f32(name)
            b64 = s.get_field(name)
            assert np.array_equal(b32, b64.astype(np.float32))
            if prec == "fp32_mixed" and name == "u":
                assert np.array_equal(b32[g.interior], a[g.interior])
            else:
                assert np.abs(b32[g.interior] - a[g.interior]).max() <= 4e-5 * (abs(base) + 4)
