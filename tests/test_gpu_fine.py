"""Nested 2 cm patches on the GPU against the CPU oracle, and the reference's
own fine-patch tests (src/fluid_core.rs:11615-11660, src/fluid_core/near.rs:
405-446, tests/near_field.rs) run on the device.

Tolerance: max |dh| <= 1e-4 m per layer on the coarse window (the pass
criterion). The patch step emulates the reference box by box, so the only
differences are the last-bit results of CUDA's expf/powf/hypotf."""
import numpy as np
import pytest

import oracle as O
import silt_b200 as G
import silt_scenes as S

pytestmark = pytest.mark.gpu
TOL_H = 1.0e-4


def four_tires(z, speed=2.0, slip=0.15):
    return [dict(x=x, z=z + dz, forward_x=0.0, forward_z=1.0, radius=0.38, width=0.2, speed=speed, slip=slip)
            for (x, dz) in ((-0.7, -1.2), (0.7, -1.2), (-0.7, 1.2), (0.7, 1.2))]


def drive(core, steps, dt, speed=2.0, z0=-1.0):
    z = np.float32(z0)
    events = []
    for _ in range(steps):
        for t in four_tires(float(z), speed):
            core.push_tire(**t)
        events.append(core.step(dt))
        z = np.float32(z + np.float32(speed) * np.float32(dt))
    return events


def compare(ref, dev, tol=TOL_H):
    out = {}
    for name in ("water", "slurry"):
        out[name] = float(np.abs(ref.get(name) - dev.get(name)).max())
    assert out["water"] <= tol and out["slurry"] <= tol, out
    return out


@pytest.mark.parametrize("pace", [0, 1, 2, 3])
def test_mean_patch_drive_matches_oracle(pace):
    """Pace 0 and 1 step the open 2 cm sheet on its awake tiles; pace 2 and 3
    split the whole wet rectangle by adaptive CFL (pace 3: one pressure solve,
    then a flux per Courant slice, pace3_slices src/fluid_core.rs:1836),
    capped at eight substeps as the reference's ThroughDrive sets it
    (src/world.rs:4307-4308)."""
    dt = 1.0 / 30.0
    ref, dev = O.Core(), G.Sheet()
    for c in (ref, dev):
        c.pour_water(-3.0, 3.0, -2.0, 8.0, 0.08)
        c.pour_slurry(-1.0, 1.0, -2.0, 6.0, 0.03, 0, 0.6)
        c.set_fine_pace(pace)
        if pace >= 2:
            c.set_fine_sub_cap(8.0)
    ev_r = drive(ref, 20, dt)
    ev_d = drive(dev, 20, dt)
    d = compare(ref, dev)
    print("max |dh|", d)
    assert sum(len(e) for e in ev_r) == sum(len(e) for e in ev_d)
    vr = sum(e[6] for es in ev_r for e in es)
    vd = sum(e[6] for es in ev_d for e in es)
    assert abs(vr - vd) <= 1e-6 + 1e-3 * vr
    assert ref.near_tiles() == dev.near_tiles()


def test_per_tire_patches_match_oracle():
    dt = 1.0 / 120.0
    scene = S.grid(res=256)
    ref = O.Core(res=256, fine_res=64, layout=1)
    dev = G.Sheet(res=256, fine_res=64, layout=G.FINE_PER_TIRE)
    for c in (ref, dev):
        S.seed_core(c, scene)
        c.set_inflow(0, -2.0, 2.0, 0.5)
    for k in range(30):
        for t in S.tires_at(k * dt, speed=5.0, z0=-5.0):
            ref.push_tire(**t)
            dev.push_tire(**t)
        ref.step(dt)
        dev.step(dt, want_spray=False)
    compare(ref, dev)
    lr, ld = ref.ledger(), dev.ledger()
    assert abs(ld["water_m3"] - lr["water64"]) <= 1e-5 * lr["water64"]


def test_fine_patch_leaves_no_hole_in_deep_water():
    dev = G.Sheet()
    dev.pour_water(-6.0, 6.0, -6.0, 6.0, 0.40)
    before = dev.ledger()["total_m3"]
    for _ in range(30):
        dev.push_tire(x=0.0, z=0.0, forward_x=0.0, forward_z=1.0, radius=0.01, width=0.01, speed=0.0, slip=0.0)
        dev.step(1.0 / 30.0, want_spray=False)
    after = dev.ledger()["total_m3"]
    assert abs(after - before) < 1.0e-3 * before
    water = dev.get("water").reshape(200, 200)
    xs = (np.arange(200) + 0.5) * 0.2 - 20.0
    X, Z = np.meshgrid(xs, xs)
    ring = (np.hypot(X, Z) >= 0.5) & (np.abs(X) <= 2.0) & (np.abs(Z) <= 2.0)
    assert water[ring].min() > 0.37


def test_detail_survives_refine_and_keeps_volume():
    dt = 1.0 / 30.0
    dev = G.Sheet()
    dev.pour_water(-2.0, 2.0, -2.0, 2.0, 0.08)
    t = dict(x=0.7, z=0.0, forward_x=0.0, forward_z=1.0, radius=0.38, width=0.2, speed=3.0, slip=0.3)
    for _ in range(6):
        dev.push_tire(**t)
        dev.step(dt, want_spray=False)
    assert dev.near_tiles() > 0
    before = dev.ledger()["water_m3"]
    fine, _ = dev.fine_water_debug([t])
    after = dev.ledger()["water_m3"]
    assert abs(after - before) < 1.0e-6
    assert (fine >= 0).all()
    f = fine.reshape(160, 160)
    spread = max(float(np.ptp(f[cj * 10:cj * 10 + 10, ci * 10:ci * 10 + 10])) for cj in range(16) for ci in range(16)
                 if f[cj * 10:cj * 10 + 10, ci * 10:ci * 10 + 10].max() > 0)
    assert spread > 1.0e-3


def test_unheld_tiles_fade_out():
    dt = 1.0 / 30.0
    dev = G.Sheet()
    dev.pour_water(-2.0, 2.0, -2.0, 2.0, 0.08)
    t = dict(x=0.7, z=0.0, forward_x=0.0, forward_z=1.0, radius=0.38, width=0.2, speed=3.0, slip=0.3)
    for _ in range(6):
        dev.push_tire(**t)
        dev.step(dt, want_spray=False)
    assert dev.near_tiles() > 0
    for _ in range(int(12.0 * 1.5 / dt)):
        dev.step(dt, want_spray=False)
    assert dev.near_tiles() == 0


def test_near_field_keeps_sub_cell_detail():
    DT, SPEED = 1.0 / 30.0, 2.0

    def run(near):
        dev = G.Sheet()
        dev.set_near_field(near)
        dev.pour_water(-3.0, 3.0, -2.0, 8.0, 0.08)
        led = dev.ledger()
        start = led["water_m3"] + led["frozen_water_m3"] + led["spray_m3"]
        drive(dev, 60, DT, SPEED)
        z = np.float32(-1.0)
        for _ in range(60):
            z = np.float32(z + np.float32(SPEED) * np.float32(DT))
        fine, _ = dev.fine_water_debug(four_tires(float(z), SPEED))
        f = fine.reshape(160, 160)
        spreads = [float(np.ptp(f[cj * 10:cj * 10 + 10, ci * 10:ci * 10 + 10])) for cj in range(16) for ci in range(16)
                   if f[cj * 10:cj * 10 + 10, ci * 10:ci * 10 + 10].max() > 1e-4]
        led = dev.ledger()
        return np.mean(spreads), led["water_m3"] + led["frozen_water_m3"] + led["spray_m3"], start

    on, off = run(True), run(False)
    assert on[0] > 1.5 * off[0], (on, off)
    for _, water, start in (on, off):
        assert abs(water - start) < 1.0e-3 * start


@pytest.mark.parametrize("engine", [G.ENGINE_WINDOW, G.ENGINE_GRID])
def test_ledger_closes_in_fp64_with_tires_and_inflow(engine):
    """Per-step conservation: water now = water before + inflow - spray - the
    volume the dry cut removes, to the f32 rounding of the cell updates. On
    the grid engine this also checks that every write outside the step (the
    inflow strip, the patch hand-back) wakes the tiles it lands in."""
    dt = 1.0 / 120.0
    scene = S.grid(res=256)
    dev = G.Sheet(res=256, fine_res=64, layout=G.FINE_PER_TIRE, engine=engine)
    S.seed_core(dev, scene)
    dev.set_inflow(0, -2.0, 2.0, 0.5)
    prev = dev.ledger()
    worst = worst_cut = 0.0
    for k in range(40):
        for t in S.tires_at(k * dt, speed=5.0, z0=-5.0):
            dev.push_tire(**t)
        dev.step(dt, want_spray=False)
        led = dev.ledger()
        expect = prev["total_m3"] + (led["opened_m3"] - prev["opened_m3"])
        worst = max(worst, abs(led["total_m3"] - expect) / expect)
        # With the dry cut's own book the FP64 books close to the f32 rounding
        # of the cell updates.
        expect_cut = expect + prev["cut_m3"]
        worst_cut = max(worst_cut, abs(led["total_m3"] + led["cut_m3"] - expect_cut) / expect_cut)
        assert led["cut_m3"] >= prev["cut_m3"]
        prev = led
    print("worst relative gap", worst, "with the cut book", worst_cut)
    assert worst < 1e-5
    assert worst_cut < 1e-6


def test_grid_engine_tracks_window_engine_with_tires():
    """The two coarse engines on the same tire drive: both step the
    reference's pair with its Gauss-Seidel confinement (the window engine box
    by box, the grid engine as a fixed point over tiles), so their depths
    agree to the pass criterion."""
    dt = 1.0 / 120.0
    scene = S.grid(res=256)
    out = []
    for engine in (G.ENGINE_WINDOW, G.ENGINE_GRID):
        dev = G.Sheet(res=256, fine_res=64, layout=G.FINE_PER_TIRE, engine=engine)
        S.seed_core(dev, scene)
        dev.set_inflow(0, -2.0, 2.0, 0.5)
        for k in range(30):
            for t in S.tires_at(k * dt, speed=5.0, z0=-5.0):
                dev.push_tire(**t)
            dev.step(dt, want_spray=False)
        out.append((dev.get("water"), dev.get("slurry")))
    assert np.abs(out[0][0] - out[1][0]).max() <= TOL_H
    assert np.abs(out[0][1] - out[1][1]).max() <= TOL_H
