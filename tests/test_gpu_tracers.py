"""The sheet's tracers on the GPU against the oracle: foam, stirred silt and
the wheel-lifted suspended solids (src/fluid_core.rs:6136-6800, :8750-9003),
the river inlet's load (:7712-7757), their window moves and their books;
and the reference's own tracer tests restated on the device
(tire_slip_stirs_a_closed_silt_book, src/fluid_core.rs:11676-11775;
wheel_cloud_settles_and_ledgers_close, tests/turbid_settle.rs:28-71).

The tracer planes are f32 cell updates in the reference's order. The device
computes e^x, x^y and hypot as the double result rounded once; the C
library's expf differs from that on ~1e-4 of inputs, and the suspended
load's settling factor e^(-dt v/h) is evaluated on every wet cell, so a run
meets such inputs. The bar is therefore bit equality with the oracle built
with the device's forms (oracle.CoreRN) and, against the default build,
1 ulp on at most a few cells (well inside the 1e-4 m of the sheet step's
parity bar). The books are FP64 sums of the reference's f32 terms, compared
with the oracle's FP64 twins: to 1e-12 relative against CoreRN and 1e-7
against the default build (a 1-ulp settling factor that the f32 column
absorbs still moves the booked landed volume by parts in 10^9)."""
import numpy as np
import pytest

import oracle as O
import silt_b200 as G
import silt_scenes as S

pytestmark = pytest.mark.gpu
F = np.float32
TRACERS = ("foam", "turbid", "susp")


def four_tires(z, speed=2.0, slip=0.15):
    return [dict(x=x, z=z + dz, forward_x=0.0, forward_z=1.0, radius=0.38, width=0.2, speed=speed, slip=slip)
            for (x, dz) in ((-0.7, -1.2), (0.7, -1.2), (-0.7, 1.2), (0.7, 1.2))]


def same_bits(a, b):
    return np.array_equal(np.asarray(a, F).view(np.uint32), np.asarray(b, F).view(np.uint32))


def check_planes(ref, dev, names=("water", "slurry", "uw", "vw") + TRACERS, ulps=0, cells=0):
    bad = {}
    for n in names:
        a, b = ref.get(n), dev.get(n)
        if same_bits(a, b):
            continue
        ia, ib = a.view(np.int32).astype(np.int64), b.view(np.int32).astype(np.int64)
        d = np.abs(ia - ib)
        if int(d.max()) > ulps or int((d != 0).sum()) > cells or (np.sign(a) != np.sign(b)).any():
            bad[n] = (float(np.abs(a - b).max()), int(d.max()), int((d != 0).sum()))
    assert not bad, bad


BOOKS = ("settled_suspended_m3", "entrained_m3", "turbid_settled_m3", "stirred_m3", "suspended_m3", "turbid_m3",
         "frozen_suspended_m3", "frozen_turbid_m3")


def check_books(ref, dev, rel):
    b, led = ref.tracer_books(), dev.ledger()
    bad = {}
    for k in BOOKS:
        want = b[k + "64"]
        if abs(led[k] - want) > rel * abs(want) + 1e-15:
            bad[k] = (led[k], want)
    assert not bad, bad


class Pair:
    """The oracle and its device-function twin driven together."""

    def __init__(self, **kw):
        self.cores = (O.Core(**kw), O.CoreRN(**kw))

    def __getattr__(self, name):
        def call(*a, **kw):
            out = [getattr(c, name)(*a, **kw) for c in self.cores]
            return out[0]
        return call

    def check(self, dev, names=("water", "slurry", "uw", "vw") + TRACERS):
        check_planes(self.cores[1], dev, names)
        check_planes(self.cores[0], dev, names, ulps=1, cells=8)
        check_books(self.cores[1], dev, 1e-12)
        check_books(self.cores[0], dev, 1e-7)


@pytest.mark.parametrize("engine", [G.ENGINE_WINDOW, G.ENGINE_GRID])
def test_tracers_match_oracle_on_a_tire_drive(engine):
    dt = 1.0 / 30.0
    ref, dev = Pair(), G.Sheet(engine=engine)
    for c in (ref, dev):
        c.pour_water(-3.0, 3.0, -2.0, 8.0, 0.08)
        c.pour_slurry(-1.0, 1.0, -2.0, 6.0, 0.03, 0, 0.6)
    z = F(-1.0)
    for k in range(24):
        if k < 16:  # the tires leave; the foam and the cloud carry on and settle
            for t in four_tires(float(z), speed=3.0, slip=0.6):
                ref.push_tire(**t)
                dev.push_tire(**t)
        ref.step(dt)
        dev.step(dt)
        z = F(z + F(3.0) * F(dt))
    ref.check(dev)
    for n in TRACERS:
        assert float(dev.get(n).max()) > 0.0, n
    fr, wr = ref.cores[1].publish()
    fd, wd = dev.publish()
    assert same_bits(wr, wd) and float(wd[3::4].max()) > 0.0


def test_turbidity_switch_and_window_move():
    """With turbidity off no solids are lifted (foam and silt remain); a window
    move parks and restores the tracers with the sheet's cells. The near field
    is off on both sides: the device releases near-field tiles that leave the
    window, the reference keeps them by world cell."""
    dt = 1.0 / 30.0
    ref, dev = Pair(), G.Sheet()
    for c in (ref, dev):
        c.set_near_field(False)
        c.set_turbidity_enabled(False)
        c.pour_water(-3.0, 3.0, -3.0, 3.0, 0.07)
    push = dict(x=0.15, z=0.2, forward_x=0.0, forward_z=1.0, radius=0.38, width=0.28, speed=8.0, slip=1.2)
    for _ in range(6):
        for c in (ref, dev):
            c.push_tire(**push)
            c.step(dt)
    assert float(dev.get("susp").max()) == 0.0 and dev.ledger()["entrained_m3"] == 0.0
    for c in (ref, dev):
        c.set_turbidity_enabled(True)
    for _ in range(4):
        for c in (ref, dev):
            c.push_tire(**push)
            c.step(dt)
    ref.check(dev)
    for cx, cz in ((0.0, 3.0), (0.0, 40.0), (0.0, 0.0)):  # a scroll, a jump away, a jump back
        ref.recenter(cx, cz)
        dev.recenter(cx, cz)
        ref.check(dev)
        led = dev.ledger()
        assert abs(led["suspended_m3"] + led["settled_suspended_m3"] + led["frozen_suspended_m3"]
                   - led["entrained_m3"]) <= 1e-9
        assert abs(led["turbid_m3"] + led["turbid_settled_m3"] + led["frozen_turbid_m3"] - led["stirred_m3"]) <= 1e-9
    for _ in range(3):
        for c in (ref, dev):
            c.push_tire(**push)
            c.step(dt)
    ref.check(dev)


def test_river_inlet_load_matches_oracle():
    """A river reach whose water arrives carrying 20% of its column as
    suspended solids, through a channel with a paddle (open water: the plume
    rides both axes and mixes)."""
    sc = S.channel()
    reach = dict(along_z=False, positive=True, cross0=-4.0, cross1=4.0, rows=4, inlet_eta=0.3, outlet_eta=0.28,
                 inlet_speed_m_s=0.75, inlet_turbidity=0.2)
    wave = dict(x0=5.0, x1=7.0, z0=-3.0, z1=3.0, dir_x=1.0, dir_z=0.0, amplitude_m_s=0.3, period_s=0.5, ramp_s=0.2)
    dev = G.Sheet(res=sc["res"], cell=sc["cell"])
    ref = Pair(threads=1)
    for c in (dev, ref):
        S.seed_basin(c, sc)
        c.set_open_water(True, 1.0, 0.035, 0.06)
        c.set_river_reach(reach)
        c.set_wave_maker(wave)
    for _ in range(40):
        dev.step(1.0 / 120.0, want_spray=False)
        ref.step(1.0 / 120.0)
    ref.check(dev, ("water", "uw", "vw", "susp", "foam"))
    assert dev.ledger()["entrained_m3"] > 0.0


def test_batch_tracers_equal_single_windows():
    scenes = [S.grid(res=r, seed=0x55 + r, puddles=3) for r in (64, 130, 200)]
    import torch

    stream = torch.cuda.Stream()
    alone, grouped = [], []
    for sc in scenes:
        for dst, st in ((alone, None), (grouped, stream.cuda_stream)):
            sh = G.Sheet(res=sc["res"], fine_res=64, layout=G.FINE_PER_TIRE, engine=G.ENGINE_GRID, stream=st)
            S.seed_core(sh, sc)
            dst.append(sh)
    batch = G.Batch(grouped)
    dt = 1.0 / 120.0
    for k in range(1, 30):
        idx, ts = [], []
        for w in range(len(scenes)):
            tires = S.tires_at(k * dt, speed=5.0, z0=-3.0)[:1 + w]
            for t in tires:
                alone[w].push_tire(**t)
                idx.append(w)
                ts.append(t)
            alone[w].step(dt, want_spray=False)
        batch.push_tires(idx, ts)
        batch.step(dt)
    for w in range(len(scenes)):
        for n in ("water", "slurry") + TRACERS:
            assert same_bits(alone[w].get(n), grouped[w].get(n)), (w, n)
        la, lb = alone[w].ledger(), batch.ledgers()[w]
        for key in ("entrained_m3", "stirred_m3", "suspended_m3", "turbid_m3", "settled_suspended_m3"):
            assert abs(la[key] - lb[key]) <= 1e-12 + 1e-9 * abs(la[key]), (w, key)
    batch.close()


PUSH = dict(x=0.15, z=0.2, forward_x=0.0, forward_z=1.0, radius=0.38, width=0.28, speed=8.0, slip=1.2)


def test_tire_slip_stirs_a_closed_silt_book():
    """src/fluid_core.rs:11676-11775 on the device (the silt book in FP64)."""
    dev = G.Sheet()
    dev.pour_water(-3.0, 3.0, -3.0, 3.0, 0.07)
    dt = 1.0 / 30.0
    for _ in range(10):
        dev.push_tire(**PUSH)
        dev.step(dt)
        led = dev.ledger()
        assert abs(led["stirred_m3"] - (led["turbid_m3"] + led["turbid_settled_m3"] + led["frozen_turbid_m3"])) < 1e-3
        assert dev.non_finite_count() == 0
    foam, turbid = dev.get("foam"), dev.get("turbid")
    assert float(turbid.max()) > 1.0e-4 and float(foam.max()) > 0.05
    film = dev.get("water") + dev.get("slurry")
    assert int(((foam != 0) & (film < 1e-5)).sum() + ((turbid != 0) & (film < 1e-5)).sum()) == 0
    stirred = dev.ledger()["stirred_m3"]
    dev.recenter(0.0, 40.0)
    dev.recenter(0.0, 0.0)
    led = dev.ledger()
    assert abs(led["stirred_m3"] - stirred) < 1e-6
    assert abs(led["stirred_m3"] - (led["turbid_m3"] + led["turbid_settled_m3"] + led["frozen_turbid_m3"])) < 1e-3


def test_wheel_cloud_settles_and_ledgers_close():
    """tests/turbid_settle.rs:28-71 on the device."""
    dt = F(1.0 / 30.0)
    dev = G.Sheet()
    assert dev.pour_water(-2.4, 2.4, -3.2, 3.4, 0.10) > 0.1
    z = F(-3.0)
    while z < F(2.4):
        dev.push_tire(x=0.0, z=float(z), forward_x=0.0, forward_z=1.0, radius=0.36, width=0.22, speed=3.0, slip=0.8)
        dev.step(float(dt))
        z = F(z + F(3.0) * dt)
    a = dev.publish()[1][3::4]
    assert np.isfinite(a).all() and a.min() >= 0.0 and a.max() <= 1.0
    peak_max, peak_sum = float(a.max()), float(a.sum(dtype=np.float32))
    assert peak_max > 0.05
    for _ in range(int(40.0 / dt)):
        dev.step(float(dt))
    late_sum = float(dev.publish()[1][3::4].sum(dtype=np.float32))
    assert late_sum < peak_sum * 0.35, (peak_sum, late_sum)
    led = dev.ledger()
    assert abs(led["suspended_m3"] + led["settled_suspended_m3"] + led["frozen_suspended_m3"]
               - led["entrained_m3"]) <= 1e-6
    assert abs(led["turbid_m3"] + led["turbid_settled_m3"] + led["frozen_turbid_m3"] - led["stirred_m3"]) <= 1e-6


def test_idle_tracer_steps_are_skipped_and_change_nothing():
    """With nothing to carry (no foam, no silt above 1e-8, no suspended load)
    and no tire or surface drive, a tracer step changes nothing; the library
    learns that from the device's report of an earlier step and then skips
    those launches until a trigger. The 200 window without tires goes idle;
    tires then wake the tracers again; the oracle runs every step throughout."""
    dt = 1.0 / 120.0
    sc = S.window200()
    ref, dev = Pair(), G.Sheet()
    for c in (ref, dev):
        S.seed_core(c, sc)
    for _ in range(12):
        for c in (ref, dev):
            c.step(dt)
    dev.set_step_timing(True)
    for _ in range(6):
        for c in (ref, dev):
            c.step(dt)
    idle = dev.step_parts()
    dev.set_step_timing(False)
    push = dict(x=0.15, z=0.2, forward_x=0.0, forward_z=1.0, radius=0.38, width=0.28, speed=8.0, slip=1.2)
    dev.set_step_timing(True)
    for _ in range(6):
        for c in (ref, dev):
            c.push_tire(**push)
            c.step(dt)
    busy = dev.step_parts()
    dev.set_step_timing(False)
    ref.check(dev)
    assert float(dev.get("foam").max()) > 0.0
    # The idle steps launched only the window engine (and no tracer kernel).
    assert idle["launches"] / 6 < busy["launches"] / 6 - 8, (idle["launches"], busy["launches"])
