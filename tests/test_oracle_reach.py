"""The river reach and the wave maker on the oracle (FluidCore::set_river_reach,
set_wave_maker; src/fluid_core.rs:7420-7480, :7638-7745): the reach "neither
mints nor deletes water" (its bank is on the ledger) and keeps the stream
running; the paddle drives the strip's water back and forth."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "dirty-gen_b200"))

import oracle  # noqa: E402
import silt_scenes as S  # noqa: E402

DT = 1.0 / 120.0
REACH = dict(along_z=False, positive=True, cross0=-4.0, cross1=4.0, rows=4, inlet_eta=0.3, outlet_eta=0.28,
             inlet_speed_m_s=0.75)


def reach_core(reach=REACH):
    c = oracle.Core(threads=1)
    S.seed_basin(c, S.channel())
    c.set_open_water(True, 1.0, 0.035, 0.06)
    c.set_river_reach(reach)
    return c


def books(c):
    l = c.ledger()
    return l["water64"] + l["slurry64"] + c.reach_bank_m3()


def test_reach_keeps_the_books_and_the_current():
    c = reach_core()
    free = oracle.Core(threads=1)
    S.seed_basin(free, S.channel())
    free.set_open_water(True, 1.0, 0.035, 0.06)
    v0 = books(c)
    for _ in range(60):
        c.step(DT)
        free.step(DT)
    assert c.reach_bank_m3() > 0.0  # the lower outlet stage banks water
    assert abs(books(c) - v0) <= 2e-5 * v0
    res = 200
    # Just downstream of the inlet rows the stream keeps its speed; in the
    # closed window it stalls against the upstream wall.
    u_reach = c.get("uw").reshape(res, res)[:, 6]
    u_free = free.get("uw").reshape(res, res)[:, 6]
    wet = c.get("water").reshape(res, res)[:, 6] > 0.05
    assert float(u_reach[wet].mean()) > float(u_free[wet].mean()) + 0.05


def test_wave_maker_drives_the_strip_back_and_forth():
    c = oracle.Core(threads=1)
    S.seed_basin(c, S.channel(speed=0.0))
    c.set_open_water(True, 1.0, 0.0, 0.0)
    c.set_wave_maker(dict(x0=5.0, x1=7.0, z0=-3.0, z1=3.0, dir_x=1.0, dir_z=0.0, amplitude_m_s=0.3, period_s=0.5,
                          ramp_s=0.0))
    res = 200
    x, z = S.cell_centres(res, 0.2, S.snap_origin(0.0, 0.0, 40.0, 0.2))
    strip = (np.abs(x - 6.0) < 0.5) & (np.abs(z) < 1.5)
    signs = []
    for k in range(60):
        c.step(DT)
        if k % 15 == 7:
            signs.append(float(c.get("uw").reshape(res, res)[strip].mean()))
    assert max(signs) > 0.05 and min(signs) < -0.05, signs
