"""The render-contract reads on the GPU against the oracle: coarse_cell
(src/fluid_core.rs:6998-7035), export_maps (:6941-6975) and the film/flow
publish (src/render_contract.rs:457-496), after a tire drive; and the
reference's own test fluid_sheet_publishes_film_and_flow
(src/render_contract.rs:1576-1608) restated.

These are per-cell formulas of the stepped state, so once the state matches
bit for bit the reads must too: the bar is bit equality, the turbidity
channel (flow.A, from the tracers' suspended load and stirred silt)
included."""
import numpy as np
import pytest

import oracle as O
import silt_b200 as G

pytestmark = pytest.mark.gpu
F = np.float32


def four_tires(z, speed=2.0, slip=0.15):
    return [dict(x=x, z=z + dz, forward_x=0.0, forward_z=1.0, radius=0.38, width=0.2, speed=speed, slip=slip)
            for (x, dz) in ((-0.7, -1.2), (0.7, -1.2), (-0.7, 1.2), (0.7, 1.2))]


def drive_pair(steps=12, dt=1.0 / 30.0):
    ref, dev = O.Core(), G.Sheet()
    for c in (ref, dev):
        c.pour_water(-3.0, 3.0, -2.0, 8.0, 0.08)
        c.pour_slurry(-1.0, 1.0, -2.0, 6.0, 0.03, 0, 0.6)
    z = F(-1.0)
    for _ in range(steps):
        for t in four_tires(float(z)):
            ref.push_tire(**t)
            dev.push_tire(**t)
        ref.step(dt)
        dev.step(dt)
        z = F(z + F(2.0) * F(dt))
    for name in ("water", "slurry", "uw", "vw", "us", "vs"):
        a, b = ref.get(name), dev.get(name)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), name
    return ref, dev


def finite0(x):
    return np.where(np.isfinite(x), x, F(0.0)).astype(F)


def film_velocity(ref):
    """coarse_cell's thickness-weighted velocity (src/fluid_core.rs:7008-7017) in float32."""
    hw, hs = finite0(ref.get("water")), finite0(ref.get("slurry"))
    film = hw + hs
    with np.errstate(invalid="ignore", divide="ignore"):
        u = finite0((ref.get("uw") * hw + ref.get("us") * hs) / film)
        v = finite0((ref.get("vw") * hw + ref.get("vs") * hs) / film)
    dry = film < F(1.0e-5)
    return np.where(dry, F(0.0), u).astype(F), np.where(dry, F(0.0), v).astype(F), hw, hs


def same_bits(a, b):
    a, b = np.asarray(a, F), np.asarray(b, F)
    return np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_publish_film_flow_matches_oracle_after_a_drive():
    ref, dev = drive_pair()
    fr, wr = ref.publish()
    fd, wd = dev.publish()
    assert same_bits(fr, fd)
    assert same_bits(wr, wd)
    assert float(wd[3::4].max()) > 0.0  # the wake's suspended load and stirred silt
    assert int((fd[0::2] > 0.01).sum()) > 100


def test_export_maps_match_the_reference_formula():
    ref, dev = drive_pair()
    m = dev.export_maps()
    bed, hw_raw, hs_raw = ref.get("bed"), ref.get("water"), ref.get("slurry")
    u, v, _, _ = film_velocity(ref)
    assert same_bits(m["height"], bed + hw_raw + hs_raw)
    assert same_bits(m["vel_u"], u)
    assert same_bits(m["vel_v"], v)
    assert same_bits(m["moisture"], ref.get("moisture"))


def test_coarse_cell_matches_the_reference_formula():
    ref, dev = drive_pair()
    res = 200
    u, v, hw, hs = film_velocity(ref)
    bed, moist = ref.get("bed"), ref.get("moisture")
    ox, oz = ref.origin()
    rng = np.random.default_rng(7)
    wet = np.flatnonzero(hw + hs > 1e-3)
    cells = list(rng.choice(wet, 40, replace=False)) + [0, res - 1, res * res - 1, 101 * res + 99]
    for idx in cells:
        i, j = int(idx % res), int(idx // res)
        c = dev.coarse_cell(i, j)
        turb = F(0.0) if hw[idx] < F(1e-5) else np.clip(
            (max(finite0(ref.get("susp")[idx]), F(0)) + max(finite0(ref.get("turbid")[idx]), F(0))) / hw[idx], 0, 1)
        want = dict(x=F(ox) + (F(i) + F(0.5)) * F(0.2), z=F(oz) + (F(j) + F(0.5)) * F(0.2),
                    bed_m=finite0(bed[idx]), water_m=hw[idx], slurry_m=hs[idx], moisture=finite0(moist[idx]),
                    u=u[idx], v=v[idx], turbidity=F(turb))
        for k, w in want.items():
            assert same_bits(F(c[k]), F(w)), (i, j, k, c[k], w)
    assert dev.coarse_cell(res, 0) is None and dev.coarse_cell(0, -1) is None


def test_fluid_sheet_publishes_film_and_flow():
    """src/render_contract.rs:1576-1608: a 6 cm pour with a spinning tire on
    it, one 1/60 s step, then the publish carries the poured film and the
    window it covers."""
    dev = G.Sheet()
    dev.pour_water(-1.5, 1.5, -1.5, 1.5, 0.06)
    dev.push_tire(x=0.0, z=0.0, forward_x=0.0, forward_z=1.0, radius=0.36, width=0.22, speed=6.0, slip=0.8)
    dev.step(1.0 / 60.0)
    film, flow = dev.publish()
    wet = int((film[0::2] > 0.01).sum())
    assert wet > 10, wet
    assert np.isfinite(flow).all()
    x0, z0, extent = dev.window_bounds()
    ox, oz = G.window_origin((0.0, 0.0))
    assert abs(x0 - ox) < 1e-4 and abs(z0 - oz) < 1e-4 and abs(extent - 40.0) < 1e-4
