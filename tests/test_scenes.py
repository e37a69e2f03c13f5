"""The synthetic scenes are seeded and have the stated shapes and ranges."""
import numpy as np

import silt_scenes as S


def test_window200_shapes_and_ranges():
    sc = S.window200()
    assert sc["bed"].shape == (200 * 200,) and sc["bed"].dtype == np.float32
    assert abs(sc["water"].max() - 0.10) < 0.005
    s = sc["slurry"][sc["slurry"] > 0]
    assert 0.02 <= s.min() and s.max() <= 0.05 and np.unique(s).size == 1
    assert np.abs(sc["bed"]).max() < 0.6
    again = S.window200()
    assert np.array_equal(sc["bed"], again["bed"]) and np.array_equal(sc["slurry"], again["slurry"])


def test_grid_has_eight_puddles_and_ruts():
    sc = S.grid(res=512)
    assert (sc["water"] > 0).sum() > 0
    assert sc["water"].max() <= 0.2
    assert (sc["slurry"] > 0).sum() > 0


def test_hash01_matches_u32_arithmetic():
    # hash01 of src/fluid_core.rs:4639 evaluated with Python integers.
    def ref(ix, iz, seed):
        n = (((ix & 0xFFFFFFFF) * 0x27BB2EE6 + (iz & 0xFFFFFFFF) * 0x165667B1) & 0xFFFFFFFF) ^ seed
        n = (n * 0x9E3779B1) & 0xFFFFFFFF
        n ^= n >> 16
        n = (n * 0x85EBCA6B) & 0xFFFFFFFF
        n ^= n >> 13
        return np.float32(n >> 8) * np.float32(1.0 / 16777216.0)
    for ix, iz, seed in [(0, 0, 1), (-5, 7, 0x9E3779B9), (123456, -98765, 42)]:
        assert S.hash01(np.array([ix]), np.array([iz]), seed)[0] == ref(ix, iz, seed)
