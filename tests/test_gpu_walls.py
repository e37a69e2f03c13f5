"""The walled sheet on the GPU (silt_set_hydro_solids) against the oracle's
restatement of the reference's walled step (src/fluid_core.rs:1879-2082 with
`solid`, the wall passes :4225-4582, solid_mask :7288-7360, step_pair's mask
and displacement :7954-8100).

Tolerance: max |dh| <= 1e-4 m per layer (the pass criterion). The wall
passes add only IEEE arithmetic in the reference's order, and the damping
factors are the reference's libm results (the host's for the water, the
once-rounded double functions for the slurry), so the planes are compared bit
for bit where the scene allows it."""
import numpy as np
import pytest

import oracle as O
import silt_b200 as G
import silt_scenes as S

pytestmark = pytest.mark.gpu
DT = 1.0 / 120.0
TOL_H = 1.0e-4

BELLY = dict(x=0.1, z=0.4, yaw=0.35, half_length=1.15, half_width=0.70, bottom_y=-1.0, top_y=2.0, contact=0)


def wheels(z=0.0, half=0.25):
    return [dict(x=x, z=z + dz, yaw=0.05, half_length=half, half_width=0.1, bottom_y=-1.0, top_y=2.0, contact=1,
                 radius=0.38, width=0.2)
            for (x, dz) in ((-0.75, -1.2), (0.75, -1.2), (-0.75, 1.2), (0.75, 1.2))]


def compare(ref, dev, names=("water", "slurry")):
    return {n: float(np.abs(ref.get(n) - dev.get(n)).max()) for n in names}


def test_walled_window200_matches_oracle():
    """Config-1 window (ruts, puddle, slurry) with a current, the belly and
    four wheel contacts standing in it, 100 steps."""
    scene = S.window200()
    ref, dev = O.Core(), G.Sheet(engine=G.ENGINE_WINDOW)
    n = scene["res"] ** 2
    for c in (ref, dev):
        S.seed_core(c, scene)
        c.map_water_velocity(np.full(n, 0.15, np.float32), np.full(n, 0.45, np.float32))
        c.set_hydro_solids([BELLY] + wheels())
    for _ in range(100):
        ref.step(DT)
        dev.step(DT, want_spray=False)
    d = compare(ref, dev, ("water", "slurry", "uw", "vw", "us", "vs"))
    print("max |d|", d)
    assert d["water"] <= TOL_H and d["slurry"] <= TOL_H
    a, b = ref.get("water"), dev.get("water")
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), float(np.abs(a - b).max())
    assert dev.non_finite_count() == 0
    lr, ld = ref.ledger(), dev.ledger()
    assert abs(ld["water_m3"] - lr["water64"]) <= 1e-6 * lr["water64"]


def test_walled_channel_current_matches_oracle_bit_for_bit():
    """A 0.6 m/s channel against the belly: the bow, the redirect to the
    flanks and the wake, 150 steps."""
    scene = S.channel(res=128, level=0.3, speed=0.6)
    ref, dev = O.Core(res=128, soften=False), G.Sheet(res=128, soften=False, engine=G.ENGINE_WINDOW)
    for c in (ref, dev):
        S.seed_basin(c, scene)
        c.set_hydro_solids([dict(BELLY, x=0.0, z=0.0, yaw=0.0)] + wheels(z=0.0))
    for _ in range(150):
        ref.step(DT)
        dev.step(DT, want_spray=False)
    for name in ("water", "uw", "vw"):
        a, b = ref.get(name), dev.get(name)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (name, float(np.abs(a - b).max()))


def test_walls_on_tire_patches_match_oracle():
    """Tires driving through water with a wheel contact at each tire: the
    2 cm patches take the walled step (their own masks, Gauss-Seidel sweep,
    projection, adaptive substeps) and restrict back."""
    dt = 1.0 / 60.0
    ref = O.Core(res=128, fine_res=64, layout=1)
    dev = G.Sheet(res=128, fine_res=64, layout=G.FINE_PER_TIRE, engine=G.ENGINE_WINDOW)
    for c in (ref, dev):
        c.pour_water(-4.0, 4.0, -6.0, 8.0, 0.12)
        c.pour_slurry(-1.5, 1.5, -6.0, 6.0, 0.03, 0, 0.6)
    for k in range(30):
        tires = S.tires_at(k * dt, speed=3.0, z0=-3.0)
        solids = [dict(x=t["x"], z=t["z"], yaw=0.0, half_length=0.22, half_width=0.1, bottom_y=-1.0, top_y=2.0,
                       contact=1) for t in tires]
        for c in (ref, dev):
            c.set_hydro_solids(solids)
            for t in tires:
                c.push_tire(**t)
        ref.step(dt)
        dev.step(dt, want_spray=False)
    d = compare(ref, dev)
    print("max |dh|", d)
    assert d["water"] <= TOL_H and d["slurry"] <= TOL_H
    lr, ld = ref.ledger(), dev.ledger()
    assert abs(ld["water_m3"] - lr["water64"]) <= 1e-5 * lr["water64"]


def test_removing_the_walls_restores_the_open_step():
    scene = S.window200()
    ref, dev = O.Core(), G.Sheet(engine=G.ENGINE_WINDOW)
    for c in (ref, dev):
        S.seed_core(c, scene)
        c.set_hydro_solids([BELLY])
    for k in range(40):
        if k == 20:
            ref.set_hydro_solids([])
            dev.set_hydro_solids([])
        ref.step(DT)
        dev.step(DT, want_spray=False)
    d = compare(ref, dev)
    assert d["water"] <= TOL_H and d["slurry"] <= TOL_H, d


def test_walls_need_the_window_engine():
    dev = G.Sheet(res=256, engine=G.ENGINE_GRID)
    with pytest.raises(G.SiltError):
        dev.set_hydro_solids([BELLY])
    dev.set_hydro_solids([])  # removing none is fine


def test_hydro_load_and_scour_match_oracle():
    """hydro_load (src/fluid_core.rs:7164-7249) and scour_contacts
    (:7364-7420) in a 0.6 m/s channel with the belly and four wheels: the
    scoured bed, slurry and moisture match bit for bit; forces, buoyancy and
    the eroded volume within 1e-5 relative (FP64 sums of the reference's f32
    terms); block counts and the deepest scour exactly. The ledger closes
    with the scoured bed booked as opened volume."""
    scene = S.channel(res=128, level=0.3, speed=0.6)
    ref, dev = O.Core(res=128, soften=False), G.Sheet(res=128, soften=False, engine=G.ENGINE_WINDOW)
    wheels = [dict(x=x, z=z, yaw=0.0, half_length=0.25, half_width=0.15, bottom_y=-1.0, top_y=2.0, contact=1,
                   radius=0.38, width=0.2) for x in (-2.0, 2.0) for z in (-1.5, 1.5)]
    for c in (ref, dev):
        S.seed_basin(c, scene)
        c.set_hydro_solids([dict(BELLY, x=0.0, z=0.0, yaw=0.0)] + wheels)
    def books(led):
        return led["total_m3"] + led["cut_m3"] - led["opened_m3"]

    prev = books(dev.ledger())
    for k in range(80):
        ref.step(DT)
        dev.step(DT, want_spray=False)
        # The books are the FP64 sums of the state, which is the oracle's bit
        # for bit; what they do not close step to step is the f32 rounding
        # of the reference's own cell updates at the walls (displaced and
        # redirected shares on ~0.4 m bow columns), ~1e-9 of the volume.
        led, lo = dev.ledger(), ref.ledger()
        assert abs(led["water_m3"] - lo["water64"]) <= 1e-12 * lo["water64"], k
        assert abs(led["slurry_m3"] - lo["slurry64"]) <= 1e-12 * max(lo["slurry64"], 1.0), k
        now = books(led)
        assert abs(now - prev) <= 4e-9 * prev, (k, now - prev)
        prev = now
        if (k + 1) % 20:
            continue
        lr, ld = ref.hydro_load(), dev.hydro_load()
        for key, floor in (("force_x", 1e-3), ("force_z", 1e-3), ("buoyancy_n", 1e-3), ("hull_buoyancy_n", 1e-3),
                           ("wheel_buoyancy_n", 1e-3), ("displaced_m3", 1e-9), ("eroded_m3", 1e-12)):
            assert abs(ld[key] - lr[key]) <= 1e-5 * abs(lr[key]) + floor, (k, key, lr[key], ld[key])
        for key in ("wheel_blocks", "belly_blocks", "hole_m"):
            assert ld[key] == lr[key], (k, key, lr[key], ld[key])
    assert lr["eroded_m3"] > 0.0 and lr["force_x"] > 0.0
    for name in ("water", "slurry", "bed", "moisture", "uw", "vw", "us", "vs"):
        a, b = ref.get(name), dev.get(name)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (name, float(np.abs(a - b).max()))
