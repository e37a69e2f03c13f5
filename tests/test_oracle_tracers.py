"""The tracers of the sheet (foam, stirred silt, wheel-lifted suspended
solids; src/fluid_core.rs:6136-6800, :8750-9003) in the oracle, pinned by the
reference's own tests restated: tire_slip_stirs_a_closed_silt_book
(src/fluid_core.rs:11676-11775) and wheel_cloud_settles_and_ledgers_close
(tests/turbid_settle.rs:28-71), with their tolerances. No GPU is needed."""
import math

import numpy as np

import oracle as O

CELL = 0.2
RES = 200


def silt_book_gap(c):
    """src/fluid_core.rs:6171-6195: |stirred - (column + settled + parked)| in f32."""
    b = c.tracer_books()
    return abs(np.float32(b["stirred_m3"]) - (np.float32(b["turbid_m3"]) + np.float32(b["turbid_settled_m3"])
                                              + np.float32(b["frozen_turbid_m3"])))


def suspended_gap(c):
    """src/fluid_core.rs:6886-6889: |column + settled + parked - entrained| in f32."""
    b = c.tracer_books()
    return abs(np.float32(b["suspended_m3"]) + np.float32(b["settled_suspended_m3"])
               + np.float32(b["frozen_suspended_m3"]) - np.float32(b["entrained_m3"]))


def foam_turbid_at(c, x, z):
    """src/fluid_core.rs:6147-6167."""
    ox, oz = c.origin()
    i, j = math.floor((x - ox) / CELL), math.floor((z - oz) / CELL)
    if i < 0 or j < 0 or i >= RES or j >= RES:
        return 0.0, 0.0
    idx = j * RES + i
    film = c.get("water")[idx] + c.get("slurry")[idx]
    if not np.isfinite(film) or film < 1e-5:
        return 0.0, 0.0
    f = c.get("foam")[idx]
    foam = 0.0 if film < 0.004 or not np.isfinite(f) else float(np.clip(f, 0.0, 1.0))
    t = c.get("turbid")[idx]
    return foam, float(max(t, 0.0)) if np.isfinite(t) else 0.0


def max_near(c, x, z, radius):
    foam = turbid = 0.0
    steps = math.ceil(radius / CELL) + 1
    for dj in range(-steps, steps + 1):
        for di in range(-steps, steps + 1):
            px, pz = x + di * CELL, z + dj * CELL
            if math.hypot(px - x, pz - z) > radius:
                continue
            f, t = foam_turbid_at(c, px, pz)
            foam, turbid = max(foam, f), max(turbid, t)
    return foam, turbid


def reference_total(c):
    """FluidLedger::total_m3 (src/fluid_core.rs:6840-6853) on the sheet path, FP64 sums."""
    led, b = c.ledger(), c.tracer_books()
    return (led["water64"] + led["slurry64"] + led["frozen_water_m3"] + led["frozen_slurry_m3"] + led["spray_m3"]
            + b["suspended_m364"] + b["settled_suspended_m364"] + b["frozen_suspended_m364"])


PUSH = dict(x=0.15, z=0.2, forward_x=0.0, forward_z=1.0, radius=0.38, width=0.28, speed=8.0, slip=1.2)


def test_tire_slip_stirs_a_closed_silt_book():
    c = O.Core()
    c.pour_water(-3.0, 3.0, -3.0, 3.0, 0.07)
    before = reference_total(c)
    dt = 1.0 / 30.0
    for _ in range(10):
        c.push_tire(**PUSH)
        c.step(dt)
        assert silt_book_gap(c) < 1.0e-3
        assert c.non_finite_count() == 0
    foam, turbid = max_near(c, PUSH["x"], PUSH["z"], 0.7)
    assert turbid > 1.0e-4, turbid
    assert foam > 0.05, foam
    assert foam_turbid_at(c, 8.0, 8.0) == (0.0, 0.0)
    film = c.get("water") + c.get("slurry")
    dry = film < 1e-5
    assert int(((c.get("foam") != 0) & dry).sum() + ((c.get("turbid") != 0) & dry).sum()) == 0
    stirred = c.tracer_books()["stirred_m3"]
    c.recenter(0.0, 40.0)
    assert silt_book_gap(c) < 1.0e-3
    c.recenter(0.0, 0.0)
    assert abs(c.tracer_books()["stirred_m3"] - stirred) < 1.0e-6
    assert silt_book_gap(c) < 1.0e-3
    after = reference_total(c) - c.tracer_books()["entrained_m364"]
    assert abs(after - before) < 1.0e-3, (before, after)
    # A tire that is not moving paints no foam disc on the wet interior.
    still = O.Core(center=(0.0, 2.0))
    still.pour_water(-2.0, 2.0, 0.0, 4.0, 0.06)
    still.push_tire(**dict(PUSH, speed=0.0, slip=0.0))
    still.step(dt)
    assert foam_turbid_at(still, PUSH["x"], PUSH["z"])[1] == 0.0
    h = still.get("water") + still.get("slurry")
    ox, oz = still.origin()
    disc = 0
    steps = math.ceil(0.7 / CELL)
    for dj in range(-steps, steps + 1):
        for di in range(-steps, steps + 1):
            px, pz = PUSH["x"] + di * CELL, PUSH["z"] + dj * CELL
            if math.hypot(px - PUSH["x"], pz - PUSH["z"]) > 0.7:
                continue
            i, j = math.floor((px - ox) / CELL), math.floor((pz - oz) / CELL)
            if not (1 <= i < RES - 1 and 1 <= j < RES - 1):
                continue
            idx = j * RES + i
            if h[idx] < 0.02 or min(h[idx - 1], h[idx + 1], h[idx - RES], h[idx + RES]) < 0.02:
                continue
            if still.get("foam")[idx] > 0 or still.get("turbid")[idx] > 0:
                disc += 1
    assert disc == 0


def test_wheel_cloud_settles_and_ledgers_close():
    """tests/turbid_settle.rs:28-71: the published turbidity (flow.A) of a
    wheel's cloud in a still pond falls below 35% of its peak sum within
    40 s, and both the suspended and the silt books close to 1e-6 m^3."""
    dt = np.float32(1.0 / 30.0)
    c = O.Core()
    assert c.pour_water(-2.4, 2.4, -3.2, 3.4, 0.10) > 0.1
    z = np.float32(-3.0)
    while z < np.float32(2.4):
        c.push_tire(x=0.0, z=float(z), forward_x=0.0, forward_z=1.0, radius=0.36, width=0.22, speed=3.0, slip=0.8)
        c.step(float(dt))
        z = np.float32(z + np.float32(3.0) * dt)
    a = c.publish()[1][3::4]
    assert np.isfinite(a).all() and a.min() >= 0.0 and a.max() <= 1.0
    peak_max, peak_sum = float(a.max()), float(np.float32(a.sum(dtype=np.float32)))
    assert peak_max > 0.05, peak_max
    for _ in range(int(40.0 / dt)):
        c.step(float(dt))
    a = c.publish()[1][3::4]
    late_sum = float(np.float32(a.sum(dtype=np.float32)))
    assert late_sum < peak_sum * 0.35, (peak_sum, late_sum)
    assert suspended_gap(c) <= 1.0e-6, suspended_gap(c)
    assert silt_book_gap(c) <= 1.0e-6, silt_book_gap(c)


def test_turbidity_switch_turns_the_suspended_load_off():
    """set_turbidity_enabled(false) (src/fluid_core.rs:5097): no wake
    entrainment and no suspended step; the stirred silt and foam remain."""
    c = O.Core()
    c.set_turbidity_enabled(False)
    c.pour_water(-3.0, 3.0, -3.0, 3.0, 0.07)
    for _ in range(5):
        c.push_tire(**PUSH)
        c.step(1.0 / 30.0)
    b = c.tracer_books()
    assert b["entrained_m3"] == 0.0 and b["suspended_m3"] == 0.0
    assert b["stirred_m3"] > 0.0


def test_device_function_build_moves_only_a_book():
    """The oracle built with e^x, x^y and hypot as the double result rounded
    once (oracle.CoreRN, the device's forms) keeps every plane of a tire drive
    bit for bit and moves only the settled-suspended book, by parts in 10^9:
    a 1-ulp settling factor from the C library's expf is absorbed by the f32
    update of the column but not by the FP64 book of what landed."""
    F = np.float32

    def drive(C):
        c = C()
        c.pour_water(-3.0, 3.0, -2.0, 8.0, 0.08)
        c.pour_slurry(-1.0, 1.0, -2.0, 6.0, 0.03, 0, 0.6)
        z = F(-1.0)
        for k in range(24):
            if k < 16:
                for x, dz in ((-0.7, -1.2), (0.7, -1.2), (-0.7, 1.2), (0.7, 1.2)):
                    c.push_tire(x=x, z=float(z + F(dz)), forward_x=0.0, forward_z=1.0, radius=0.38, width=0.2,
                                speed=3.0, slip=0.6)
            c.step(1.0 / 30.0)
            z = F(z + F(3.0) * F(1.0 / 30.0))
        return c

    a, b = drive(O.Core), drive(O.CoreRN)
    for n in ("water", "slurry", "uw", "vw", "foam", "turbid", "susp"):
        assert np.array_equal(a.get(n).view(np.uint32), b.get(n).view(np.uint32)), n
    ba, bb = a.tracer_books(), b.tracer_books()
    for k in O.TRACER_BOOKS:
        rel = abs(ba[k + "64"] - bb[k + "64"]) / max(abs(ba[k + "64"]), 1e-30)
        assert rel < 1e-8, (k, rel)
