"""Window moves on the oracle (FluidCore::recenter, src/fluid_core.rs:5409-5421:
"Cells that slide off are parked. Cells that slide on are restored. The sum
does not change."), the scroll form (whole-cell moves, :9024) and the hash
form (:9147)."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "dirty-gen_b200"))

import oracle  # noqa: E402
import silt_scenes as S  # noqa: E402

DT = 1.0 / 120.0
PLANES = ("water", "slurry", "uw", "vw", "us", "vs", "moisture")


def core(steps=3):
    c = oracle.Core(threads=1)
    S.seed_core(c, S.window200())
    for _ in range(steps):
        c.step(DT)
    return c


def total(c):
    l = c.ledger()
    return l["water64"] + l["slurry64"] + l["frozen_water_m3"] + l["frozen_slurry_m3"]


def test_scroll_parks_and_restores_the_same_state():
    c = core()
    before = {k: c.get(k).copy() for k in PLANES}
    v0 = total(c)
    c.recenter(3.1, -2.2)  # whole cells: the scroll form
    assert c.origin() == (-17.0, np.float32(-22.2).item())
    assert c.parked_count() > 0
    assert abs(total(c) - v0) <= 1e-6 * v0
    c.recenter(0.0, 0.0)
    assert c.parked_count() == 0 and c.origin() == (-20.0, -20.0)
    for k in PLANES:
        assert np.array_equal(c.get(k), before[k]), k


def test_scroll_moves_cells_by_their_world_position():
    c = core()
    w = c.get("water").reshape(200, 200)
    c.recenter(1.0, 0.6)  # 5 cells in x, 3 in z
    w2 = c.get("water").reshape(200, 200)
    assert np.array_equal(w2[:-3, :-5], w[3:, 5:])


def test_hash_jump_parks_everything_and_comes_back():
    c = core()
    before = {k: c.get(k).copy() for k in PLANES}
    v0 = total(c)
    c.recenter(100.0, 37.0)  # no overlap
    assert float(c.get("water").max()) == 0.0 and float(c.get("slurry").max()) == 0.0
    assert abs(total(c) - v0) <= 1e-6 * v0
    c.recenter(0.0, 0.0)
    assert c.parked_count() == 0
    for k in PLANES:
        assert np.array_equal(c.get(k), before[k]), k


def test_steps_between_moves_keep_the_books():
    c = core()
    v0 = total(c)
    for k, (cx, cz) in enumerate([(2.0, 0.0), (2.0, 3.0), (-1.0, 3.0), (0.0, 0.0)]):
        c.recenter(cx, cz)
        for _ in range(4):
            c.step(DT)
    assert abs(total(c) - v0) <= 2e-4 * v0  # the dry cut's films are the only loss
