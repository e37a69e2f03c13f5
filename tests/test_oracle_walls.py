"""The oracle's walled sheet (src/fluid_core.rs:1879-2082 with `solid`, the
wall passes :4225-4582, solid_mask :7288-7360): behaviour the reference's
creek test relies on (tests/creek.rs:590-597: the water book closes to 1e-3
m^3 with wheels and belly in a current), restated on the sheet alone. The
reference has no golden vectors for this path; these properties, and the
GPU parity tests against this restatement, are what pins it."""
import numpy as np
import pytest

import oracle as O
import silt_scenes as S

DT = 1.0 / 120.0
BELLY = dict(x=0.0, z=0.0, yaw=0.3, half_length=1.15, half_width=0.70, bottom_y=-1.0, top_y=2.0, contact=0)


def channel_core(solids, res=96):
    scene = S.channel(res=res, level=0.3, speed=0.6)
    core = O.Core(res=res, soften=False)
    S.seed_basin(core, scene)
    core.set_hydro_solids(solids)
    return core, scene


def reachable_wall(mask, res):
    """Wall cells with an open cell within two cells: displacement empties
    them (a column with nowhere to go stays, src/fluid_core.rs:4420-4432)."""
    m = mask.reshape(res, res) > 0
    pad = np.pad(~m, 2, constant_values=False)
    near_open = np.zeros_like(m)
    for dj in range(5):
        for di in range(5):
            near_open |= pad[dj:dj + res, di:di + res]
    return (m & near_open).ravel()


def cell_index(core, scene, x, z):
    o = scene["origin"]
    return int((z - o[1]) / 0.2) * core.res + int((x - o[0]) / 0.2)


def test_mask_draws_walls_then_contacts_and_needs_water_above_the_underside():
    wheel = dict(x=0.8, z=0.0, yaw=0.0, half_length=0.3, half_width=0.3, bottom_y=-1.0, top_y=2.0, contact=1)
    core, scene = channel_core([BELLY, wheel])
    m = core.solid_mask()
    assert (m == 2).sum() > 50 and (m == 1).sum() > 4
    # The contact wins the cells it shares with the belly.
    assert m[cell_index(core, scene, 0.75, 0.0)] == 1
    assert m[cell_index(core, scene, -0.5, 0.0)] == 2
    # A body whose underside is above the surface is no wall.
    high = dict(BELLY, bottom_y=0.5)
    core.set_hydro_solids([high])
    assert core.solid_mask().sum() == 0


def test_walls_stay_dry_and_the_water_book_closes():
    core, scene = channel_core([BELLY])
    v0 = core.ledger()["water64"]
    for _ in range(59):
        core.step(DT)
    m = core.solid_mask()  # the mask the next step uses
    core.step(DT)
    w = core.get("water")
    edge = reachable_wall(m, core.res)
    assert edge.sum() > 20
    assert float(w[edge].max()) == 0.0
    v1 = core.ledger()["water64"]
    assert abs(v1 - v0) <= 1e-6 * v0, (v0, v1)
    assert core.non_finite_count() == 0


def test_current_piles_a_bow_upstream_and_a_hole_downstream():
    core, scene = channel_core([dict(BELLY, yaw=0.0, half_length=0.4, half_width=0.8)])
    for _ in range(120):
        core.step(DT)
    w = core.get("water").reshape(core.res, core.res)
    o = scene["origin"]
    row = int((0.0 - o[1]) / 0.2)
    up = int((-0.9 - o[0]) / 0.2)    # current along +x: upstream is -x
    down = int((0.9 - o[0]) / 0.2)
    assert w[row, up] > w[row, down] + 0.01, (w[row, up], w[row, down])


def test_displaced_water_goes_to_open_neighbours():
    """A wall laid over standing water: the covered columns move to the open
    cells around it and the volume stays."""
    scene = S.channel(res=64, level=0.3, speed=0.0)
    core = O.Core(res=64, soften=False)
    S.seed_basin(core, scene)
    v0 = core.ledger()["water64"]
    core.set_hydro_solids([dict(BELLY, half_length=0.5, half_width=0.3)])
    m = core.solid_mask()
    core.step(DT)
    w = core.get("water")
    assert float(w[reachable_wall(m, 64)].max()) == 0.0
    assert abs(core.ledger()["water64"] - v0) <= 1e-6 * v0


WHEEL = dict(yaw=0.0, half_length=0.25, half_width=0.15, bottom_y=-1.0, top_y=2.0, contact=1, radius=0.38, width=0.2)


def test_current_loads_the_walls_downstream_and_scours_beside_contacts():
    """hydro_load (src/fluid_core.rs:7164-7249) in a +x current: the bow
    upstream and the dynamic pressure push the bodies along +x; wheels in
    water float on their submerged segments; scour_contacts (:7364-7420)
    cuts the bed beside the contacts into the slurry as silt."""
    wheels = [dict(WHEEL, x=x, z=z) for x in (-2.0, 2.0) for z in (-1.5, 1.5)]
    core, scene = channel_core([dict(BELLY, yaw=0.0)] + wheels)
    bed0 = core.get("bed").copy()
    for _ in range(60):
        core.step(DT)
    load = core.hydro_load()
    assert load["force_x"] > 10.0 * abs(load["force_z"]), load
    assert load["wheel_blocks"] > 0 and load["belly_blocks"] > 0
    assert load["wheel_buoyancy_n"] > 0.0 and load["hull_buoyancy_n"] > 0.0
    assert abs(load["buoyancy_n"] - load["wheel_buoyancy_n"] - load["hull_buoyancy_n"]) <= 1e-3 * load["buoyancy_n"]
    assert load["eroded_m3"] > 0.0 and 0.0 < load["hole_m"] <= 0.08
    drop = bed0 - core.get("bed")
    assert float(drop.max()) == pytest.approx(load["hole_m"], rel=1e-6)
    assert abs(float(drop.astype(np.float64).sum()) * 0.04 - load["eroded_m3"]) <= 1e-5 * load["eroded_m3"] + 1e-9
    assert (core.grain()[drop > 0] == 1).all()
