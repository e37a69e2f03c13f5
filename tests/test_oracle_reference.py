"""The reference's own unit tests, restated against the CPU oracle.

These pin the restatement to the reference's behaviour: every assertion below
is the reference test's assertion, with its seeds, sizes and tolerances
(src/fluid_core.rs:11126-11817, src/fluid_core/near.rs:349-447,
tests/near_field.rs). No GPU is needed.
"""
import os

import numpy as np
import pytest

import oracle as O
from xorshift import XorShift

F = np.float32
CLAY, SILT, SAND, WATER, OTHER = 0, 1, 2, 3, 4


def column_sum(h, cell):
    """src/fluid_core.rs:4617: sequential f32 sum of max(h, 0) times the area."""
    s = F(-0.0)
    for x in np.maximum(h, F(0)):
        s = F(s + x)
    return F(s * F(F(cell) * F(cell)))


# src/fluid_core.rs:11230-11270 run_bodies_match_the_flood_fill
def test_run_bodies_match_the_flood_fill():
    rnd = XorShift(0x9E3779B9).next
    for case in range(160):
        res = [16, 40, 100, 160][case % 4]
        h = np.zeros(res * res, F)
        blobs = 1 + int(rnd() * F(12.0))
        jj, ii = np.mgrid[0:res, 0:res]
        for _ in range(blobs):
            cx = rnd() * F(res)
            cz = rnd() * F(res)
            r = F(1.0) + rnd() * F(res) * F(0.2)
            dx = ii.astype(F) - cx
            dz = jj.astype(F) - cz
            inside = ((dx * dx + dz * dz) < r * r).ravel()
            for idx in np.nonzero(inside)[0]:
                if rnd() > F(0.15):
                    h[idx] = F(0.01) + rnd() * F(0.1)
        if case % 7 == 0:
            for idx in range(res * res):
                if rnd() < F(0.3):
                    h[idx] = F(0.02)
        want = O.sheet_work_boxes(h, res, 1.0e-4, True, flood=True)
        got = O.sheet_work_boxes(h, res, 1.0e-4, True, flood=False)
        assert want == got, f"case {case}"


# src/fluid_core.rs:11272-11365 transport_open_rows_match_the_serial_edges
def test_transport_open_rows_match_the_serial_edges():
    rnd = XorShift(0x2545F491).next
    for case in range(96):
        res = [12, 37, 64, 160][case % 4]
        n = res * res
        h = np.zeros(n, F)
        vel = np.zeros(n, F)
        gate = np.ones(n, np.uint8)
        bed = np.zeros(n, F)
        for idx in range(n):
            r = rnd()
            if r < F(0.25):
                h[idx] = 0.0
            elif r < F(0.3):
                h[idx] = F(5.0e-7)
            elif r < F(0.33):
                h[idx] = F(5.0e-9)
            else:
                h[idx] = rnd() * F(0.3)
            q = rnd()
            if q < F(0.15):
                vel[idx] = 0.0
            elif q < F(0.2):
                vel[idx] = (rnd() - F(0.5)) * F(3.0e-5)
            else:
                vel[idx] = (rnd() - F(0.5)) * F(6.0)
            gate[idx] = 1 if rnd() > F(0.2) else 0
            bed[idx] = (rnd() - F(0.5)) * F(0.05)
        i0 = int(rnd() * F(3.0))
        j0 = int(rnd() * F(3.0))
        i1 = res - 1 - int(rnd() * F(3.0))
        j1 = res - 1 - int(rnd() * F(3.0))
        cell = F(0.02) + rnd() * F(0.2)
        dt = F(0.002) + rnd() * F(0.03)
        for along_x in (True, False):
            for with_bed in (False, True):
                b = bed if with_bed else None
                h_ref = h.copy()
                h_new = h.copy()
                rr, ar = O.transport_open(h_ref, vel, gate, res, cell, dt, (i0, i1, j0, j1), along_x, b, serial=True)
                rn, an = O.transport_open(h_new, vel, gate, res, cell, dt, (i0, i1, j0, j1), along_x, b, serial=False)
                assert np.array_equal(h_ref.view(np.uint32), h_new.view(np.uint32)), f"depth case {case}"
                assert np.array_equal(rr.view(np.uint32), rn.view(np.uint32)), f"removed case {case}"
                assert np.array_equal(ar.view(np.uint32), an.view(np.uint32)), f"added case {case}"


# src/fluid_core.rs:11367-11397
def test_slope_accelerates_downhill():
    res, cell = 16, 0.10
    n = res * res
    h = np.full(n, 0.05, F)
    u = np.zeros(n, F)
    v = np.zeros(n, F)
    bed = np.array([F(-0.04) * F(j) for j in range(res) for _ in range(res)], F)
    nu = np.full(n, 40.0, F)
    gate = np.ones(n, np.uint8)
    O.step_sheet(h, u, v, bed, nu, gate, res, cell, 0.05, 0.0)
    assert v[8 * res + 8] > 0.002


# src/fluid_core.rs:11399-11410
def test_viscosity_orders_clay_silt_sand_and_thins():
    clay = O.dynamic_viscosity(CLAY, 0.55)
    silt = O.dynamic_viscosity(SILT, 0.55)
    sand = O.dynamic_viscosity(SAND, 0.55)
    assert clay > silt * 1.8
    assert silt > sand * 1.5
    stiff = O.dynamic_viscosity(CLAY, 0.30)
    mid = O.dynamic_viscosity(CLAY, 0.55)
    thin = O.dynamic_viscosity(CLAY, 0.85)
    assert stiff > mid > thin


# src/fluid_core.rs:11412-11438
def test_rut_heal_times_match_the_mix():
    clay = O.rut_heal(CLAY, 0.55)
    silt = O.rut_heal(SILT, 0.55)
    thin = O.rut_heal(CLAY, 0.90)
    assert 10.0 <= clay["level_s"] <= 15.0, clay
    assert 10.0 <= silt["level_s"] <= 15.0, silt
    assert 1.0 <= thin["level_s"] <= 3.0, thin
    assert clay["still_deep_at_8s"]
    assert silt["still_deep_at_8s"]


# src/fluid_core.rs:11440-11502
def test_sheet_conserves_and_runs_downhill():
    res, cell = 24, 0.2
    n = res * res
    h = np.zeros(n, F)
    u = np.zeros(n, F)
    v = np.zeros(n, F)
    bed = np.zeros(n, F)
    nu = np.full(n, O.dynamic_viscosity(CLAY, 0.55), F)
    gate = np.ones(n, np.uint8)
    for j in range(res):
        for i in range(res):
            bed[j * res + i] = F(-0.16) * F(j)
            if 4 <= j < 9 and 8 <= i < 16:
                h[j * res + i] = 0.10

    def centroid(h):
        m = mj = F(0)
        for j in range(res):
            for i in range(res):
                s = h[j * res + i]
                m = F(m + s)
                mj = F(mj + s * F(j))
        return F(0) if m <= 1e-6 else mj / m

    before = column_sum(h, cell)
    c0 = centroid(h)
    sc = O.Scratch()
    for _ in range(60):
        O.step_sheet(h, u, v, bed, nu, gate, res, cell, 0.05, 0.02, scratch=sc)
    after = column_sum(h, cell)
    c1 = centroid(h)
    assert abs(after - before) < 1.0e-3
    assert c1 > c0 + 1.5


def still_tire(**kw):
    t = dict(x=0.0, z=0.0, forward_x=0.0, forward_z=1.0, radius=0.01, width=0.01, speed=0.0, slip=0.0)
    t.update(kw)
    return t


# src/fluid_core.rs:11615-11660
def test_fine_patch_leaves_no_hole_in_deep_water():
    core = O.Core()
    core.pour_water(-6.0, 6.0, -6.0, 6.0, 0.40)
    before = core.ledger()["water_m3"]
    for _ in range(30):
        core.push_tire(**still_tire())
        core.step(1.0 / 30.0)
    after = core.ledger()["water_m3"]
    assert abs(after - before) < 1.0e-3 * before
    lowest = 1e9
    z = F(-2.0)
    while z <= 2.0:
        x = F(-2.0)
        while x <= 2.0:
            if np.hypot(x, z) >= 0.5:
                lowest = min(lowest, core.sample(float(x), float(z))["water_m"])
            x = F(x + F(0.1))
        z = F(z + F(0.1))
    assert lowest > 0.37, lowest


def tire(x, z=0.0, speed=3.0):
    return dict(x=x, z=z, forward_x=0.0, forward_z=1.0, radius=0.38, width=0.2, speed=speed, slip=0.3)


# src/fluid_core/near.rs:405-427 (the refine/restrict round trip through fine_water_debug)
def test_detail_survives_refine_and_keeps_volume():
    dt = 1.0 / 30.0
    core = O.Core()
    core.pour_water(-2.0, 2.0, -2.0, 2.0, 0.08)
    for _ in range(6):
        core.push_tire(**tire(0.7))
        core.step(dt)
    assert core.near_tiles() > 0
    before = core.ledger()["water_m3"]
    fine, _ = core.fine_water_debug([tire(0.7)])
    after = core.ledger()["water_m3"]
    assert abs(after - before) < 1.0e-6
    assert (fine >= 0.0).all()
    sub = 10
    spread = 0.0
    for cj in range(16):
        for ci in range(16):
            blk = fine.reshape(160, 160)[cj * sub:(cj + 1) * sub, ci * sub:(ci + 1) * sub]
            if blk.max() > 0:
                spread = max(spread, float(blk.max() - blk.min()))
    assert spread > 1.0e-3, spread


# src/fluid_core/near.rs:429-446
def test_unheld_tiles_fade_out():
    dt = 1.0 / 30.0
    core = O.Core()
    core.pour_water(-2.0, 2.0, -2.0, 2.0, 0.08)
    for _ in range(6):
        core.push_tire(**tire(0.7))
        core.step(dt)
    assert core.near_tiles() > 0
    for _ in range(int(12.0 * 1.5 / dt)):
        core.step(dt)
    assert core.near_tiles() == 0


def four_tires(z, speed):
    return [dict(x=x, z=z + dz, forward_x=0.0, forward_z=1.0, radius=0.38, width=0.2, speed=speed, slip=0.15)
            for (x, dz) in ((-0.7, -1.2), (0.7, -1.2), (-0.7, 1.2), (0.7, 1.2))]


# tests/near_field.rs:45-124, with the window held still (the drive stays inside it).
@pytest.mark.parametrize("dummy", [0])
def test_near_field_keeps_sub_cell_detail(dummy):
    DT, SPEED = 1.0 / 30.0, 2.0

    def drive(near):
        core = O.Core()
        core.set_near_field(near)
        core.pour_water(-3.0, 3.0, -2.0, 8.0, 0.08)
        led = core.ledger()
        start = led["water_m3"] + led["frozen_water_m3"] + led["spray_m3"]
        z = F(-1.0)
        for _ in range(60):
            for t in four_tires(float(z), SPEED):
                core.push_tire(**t)
            core.step(DT)
            z = F(z + F(SPEED) * F(DT))
        fine, _ = core.fine_water_debug(four_tires(float(z), SPEED))
        f = fine.reshape(160, 160)
        tot = 0.0
        cnt = 0
        for cj in range(16):
            for ci in range(16):
                blk = f[cj * 10:(cj + 1) * 10, ci * 10:(ci + 1) * 10]
                if blk.max() > 1e-4:
                    tot += float(blk.max() - blk.min())
                    cnt += 1
        led = core.ledger()
        return tot / max(cnt, 1), led["water_m3"] + led["frozen_water_m3"] + led["spray_m3"], start

    on = drive(True)
    off = drive(False)
    assert on[0] > 1.5 * off[0], (on, off)
    for spread, water, start in (on, off):
        assert abs(water - start) < 1.0e-3 * start


# src/fluid_core/near.rs:353-372 floor_scale / recentre are exercised through the
# refine/restrict round trip above; the soften_border band is pinned here.
def test_soften_border_keeps_interior():
    res = 200
    u = np.ones(res * res, F)
    v = np.ones(res * res, F)
    O.lib().oracle_soften_border(u.ctypes.data, v.ctypes.data, res)
    u2 = u.reshape(res, res)
    assert u2[100, 100] == 1.0 and u2[0, 100] == 0.0
    edge = res // 12
    t = F(1) / F(edge)
    assert u2[1, 100] == t * t * (F(3) - F(2) * t)
    assert u2[edge, edge] == 1.0


def test_native_build_gives_the_portable_builds_bits(tmp_path):
    """The timed CPU baseline loads the oracle built -O3 -march=native (still
    without contraction); it must step the reference's window to the same
    bits as the portable -O2 build the parity tests use."""
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    prog = (
        "import sys, numpy as np\n"
        f"sys.path[:0] = [{os.path.join(root, 'oracle')!r}, {os.path.join(root, 'dirty-gen_b200')!r}]\n"
        "import oracle, silt_scenes as S\n"
        "if sys.argv[1] == 'native': assert oracle.use_native_build().startswith('-O3')\n"
        "sc = S.window200(); c = oracle.Core(); S.seed_core(c, sc)\n"
        "for _ in range(20): c.step(1 / 120)\n"
        "np.save(sys.argv[2], np.stack([c.get(n) for n in ('water', 'slurry', 'uw', 'vw', 'us', 'vs')]))\n")
    outs = []
    for kind in ("native", "port"):
        path = str(tmp_path / f"{kind}.npy")
        subprocess.run([sys.executable, "-c", prog, kind, path], check=True, timeout=600)
        outs.append(np.load(path))
    assert np.array_equal(outs[0].view(np.uint32), outs[1].view(np.uint32))
