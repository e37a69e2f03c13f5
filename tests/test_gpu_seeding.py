"""Seeding entries on the GPU against the oracle: lay_slurry_on_water
(src/fluid_core.rs:5236-5254) sets the slurry of every wet cell and returns
the reference's f32 volume; the step after it matches the oracle."""
import numpy as np
import pytest

import oracle as O
import silt_b200 as G
import silt_scenes as S

pytestmark = pytest.mark.gpu
DT = 1.0 / 120.0


def test_lay_slurry_on_water_matches_oracle():
    scene = S.window200()
    ref, dev = O.Core(), G.Sheet(engine=G.ENGINE_WINDOW)
    for c in (ref, dev):
        S.seed_core(c, scene)
    vr = ref.lay_slurry_on_water(0.03, 1)
    vd = dev.lay_slurry_on_water(0.03, 1)
    assert vr > 0.0 and vd == vr, (vr, vd)
    assert dev.lay_slurry_on_water(-1.0, 1) == 0.0
    for name in ("slurry", "moisture"):
        a, b = ref.get(name), dev.get(name)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), name
    for _ in range(20):
        ref.step(DT)
        dev.step(DT, want_spray=False)
    for name in ("water", "slurry", "us", "vs"):
        a, b = ref.get(name), dev.get(name)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (name, float(np.abs(a - b).max()))
