"""Parity of the CUDA sheet step with the CPU oracle (the restated reference).

Tolerance (from the build's pass criteria): max |dh| <= 1e-4 m per layer after
100 steps. The window engine (windows up to 512 cells) steps box by box with
the reference's Gauss-Seidel confinement, and the grid engine (any size)
solves the same sweep as a fixed point. The water layer's damping factor
is computed on the host with the reference's libm; the slurry's powf and expf
are the double-precision functions rounded once, which agree with the C
library's on all but a few inputs in 10^4, so on these scenes both layers
match bit for bit. The grid engine's snapshot form (the reference's
free-operator confinement) stays selectable.
"""
import numpy as np
import pytest

import oracle as O
import silt_b200 as G
import silt_scenes as S

pytestmark = pytest.mark.gpu
DT = 1.0 / 120.0
TOL_H = 1.0e-4


def run_pair(steps, scene, check_every=0, engine=G.ENGINE_AUTO):
    ref = O.Core()
    dev = G.Sheet(engine=engine)
    S.seed_core(ref, scene)
    S.seed_core(dev, scene)
    worst = []
    for k in range(steps):
        ref.step(DT)
        dev.step(DT, want_spray=False)
        if check_every and (k + 1) % check_every == 0:
            worst.append(max(np.abs(ref.get("water") - dev.get("water")).max(),
                             np.abs(ref.get("slurry") - dev.get("slurry")).max()))
    return ref, dev, worst


def test_window200_100_steps_depth_parity():
    scene = S.window200()
    ref, dev, worst = run_pair(100, scene, check_every=10)
    dw = np.abs(ref.get("water") - dev.get("water")).max()
    ds = np.abs(ref.get("slurry") - dev.get("slurry")).max()
    print(f"max |dh| water {dw:.3e} slurry {ds:.3e} trace {worst}")
    assert dw <= TOL_H and ds <= TOL_H
    # Velocities follow the same physics; they are not the pass criterion.
    for name in ("uw", "vw", "us", "vs"):
        assert np.abs(ref.get(name) - dev.get(name)).max() < 5e-3, name
    assert dev.non_finite_count() == 0


def test_window200_water_is_bit_exact_after_100_steps():
    scene = S.window200()
    ref, dev, _ = run_pair(100, scene)
    a, b = ref.get("water"), dev.get("water")
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), float(np.abs(a - b).max())
    for name in ("uw", "vw"):
        a, b = ref.get(name), dev.get(name)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (name, float(np.abs(a - b).max()))


def test_window200_slurry_is_bit_exact_after_100_steps():
    scene = S.window200()
    ref, dev, _ = run_pair(100, scene)
    for name in ("slurry", "us", "vs"):
        a, b = ref.get(name), dev.get(name)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (name, float(np.abs(a - b).max()))


def test_grid_engine_window200_within_tolerance():
    scene = S.window200()
    ref, dev, _ = run_pair(100, scene, engine=G.ENGINE_GRID)
    for name in ("water", "slurry"):
        assert np.abs(ref.get(name) - dev.get(name)).max() <= TOL_H, name


def test_window200_ledger_matches_oracle_in_fp64():
    scene = S.window200()
    ref, dev, _ = run_pair(20, scene)
    lr = ref.ledger()
    ld = dev.ledger()
    assert abs(ld["water_m3"] - lr["water64"]) <= 1e-6 * lr["water64"]
    assert abs(ld["slurry_m3"] - lr["slurry64"]) <= 1e-6 * lr["slurry64"]


def test_grid_engine_water_is_bit_exact_on_a_jacobi_sized_box():
    """The grid engine's snapshot form (SILT_CONFINE_SNAPSHOT) on a pond wider
    than 48 x 32 cells, against the oracle's pair with the free operator's
    threading: the reference then confines from a snapshot too (force_gravity_par, src/fluid_core.rs:2229-2231) and the
    water damping factor is computed on the host with the reference's libm, so
    every operation is the reference's own IEEE sequence and the depths must
    match bit for bit."""
    scene = S.window200()
    ref = O.Core(inner_par=True)
    dev = G.Sheet(engine=G.ENGINE_GRID)
    dev.set_confinement(G.CONFINE_SNAPSHOT)
    for core in (ref, dev):
        core.map_water_bed(scene["bed"], np.zeros_like(scene["water"]))
        core.pour_water(-7.0, 7.0, -7.0, 7.0, 0.06)
        core.read_substrate(scene["bed"], scene["moisture"], scene["grain"])
    for k in range(5):
        ref.step(DT)
        dev.step(DT, want_spray=False)
        a, b = ref.get("water"), dev.get("water")
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (k, float(np.abs(a - b).max()))


def test_grid_engine_device_substep_count_is_exact():
    """A fast start (15 m/s water) needs two substeps, which the grid engine
    decides on the device without waiting: the host launches three from its
    speed bound and the water layer copies itself through the third. The slurry
    pool, slow, takes one substep and copies itself through two. With two
    substeps the cells the first one wets sit two cells inside the reference's
    work box, where the box edge reaches their pressure solve, so the grid
    engine (which has no box edge) differs there by float rounding (~3e-8 m);
    a wrong substep count would move the pond's rim by ~1e-3 m."""
    scene = S.window200()
    ref = O.Core()
    dev = G.Sheet(engine=G.ENGINE_GRID)
    dev.set_step_timing(True)
    n = scene["water"].size
    fast_u = np.full(n, 15.0, np.float32)
    fast_v = np.full(n, -2.0, np.float32)
    for core in (ref, dev):
        core.map_water_bed(scene["bed"], np.zeros_like(scene["water"]))
        core.pour_water(-7.0, 7.0, -7.0, 7.0, 0.06)
        core.pour_slurry(10.0, 13.0, 10.0, 13.0, 0.03, 0, 0.55)
        core.read_substrate(scene["bed"], scene["moisture"], scene["grain"])
        core.map_water_velocity(fast_u, fast_v)
    for k in range(4):
        ref.step(DT)
        dev.step(DT, want_spray=False)
        assert np.abs(ref.get("water") - dev.get("water")).max() <= 1.0e-6, k
        assert np.abs(ref.get("slurry") - dev.get("slurry")).max() <= TOL_H, k
    assert dev.step_parts()["device_counts"] >= 1
    ld, lr = dev.ledger(), ref.ledger()
    assert abs(ld["water_m3"] - lr["water64"]) <= 1e-6 * lr["water64"]
    assert abs(ld["slurry_m3"] - lr["slurry64"]) <= 1e-6 * lr["slurry64"]


@pytest.mark.parametrize("res,cell,dt,vort", [(48, 0.06, 0.05, 0.0), (96, 0.2, 0.05, 0.02), (160, 0.1, 0.02, 0.08)])
def test_free_step_sheet_matches_oracle(res, cell, dt, vort):
    import torch
    rng = np.random.default_rng(res)
    n = res * res
    jj, ii = np.mgrid[0:res, 0:res]
    bed = (-0.03 * jj + 0.02 * np.sin(ii * 0.3)).astype(np.float32).ravel()
    h = np.where(((ii - res / 2) ** 2 + (jj - res / 3) ** 2) < (res / 5) ** 2, 0.05, 0.0).astype(np.float32).ravel()
    h += np.where(rng.random(n) < 0.05, 0.01, 0.0).astype(np.float32)
    nu = np.full(n, O.dynamic_viscosity(0, 0.55), np.float32)
    nu[: n // 2] = 0.9
    gate = np.ones(n, np.uint8)
    u = np.zeros(n, np.float32)
    v = np.zeros(n, np.float32)
    ref = [h.copy(), u.copy(), v.copy()]
    sc = O.Scratch()
    dev = [torch.tensor(x, device="cuda") for x in (h, u, v, bed, nu)]
    dgate = torch.tensor(gate, device="cuda")
    scratch = torch.zeros(G.lib().silt_step_sheet_scratch_bytes(res) // 4 + 16, dtype=torch.float32, device="cuda")
    for _ in range(20):
        O.step_sheet(ref[0], ref[1], ref[2], bed, nu, gate, res, cell, dt, vort, scratch=sc)
        G.step_sheet_device(dev[0].data_ptr(), dev[1].data_ptr(), dev[2].data_ptr(), dev[3].data_ptr(),
                            dev[4].data_ptr(), dgate.data_ptr(), res, cell, dt, vort, scratch.data_ptr())
    torch.cuda.synchronize()
    dh = np.abs(dev[0].cpu().numpy() - ref[0]).max()
    assert dh <= TOL_H, dh


@pytest.mark.parametrize("engine", [G.ENGINE_WINDOW, G.ENGINE_GRID])
def test_open_water_and_surface_diffusion_match_oracle(engine):
    """Open-water mode (mobility 1, Manning 0.035, eddy 0.06 m^2/s, the ford
    reach's settings, src/ford.rs:338-343) and surface diffusion 0.024 m^2/s on
    a basin with a 0.75 m/s current: depth within the 1e-4 m criterion after
    60 steps, velocity within 1e-3 m/s (Manning's powf and hypotf may differ
    from glibc's by an ulp), and the FP64 books closed. The grid engine runs
    against the oracle's snapshot-confinement form."""
    sc = S.basin()
    dev = G.Sheet(res=sc["res"], cell=sc["cell"], engine=engine)
    # The grid engine confines from a snapshot: the oracle's pair with the
    # free operator's form does too on boxes of at least 48 x 32 (the basin's).
    ref = O.Core(threads=1)
    for c in (dev, ref):
        S.seed_basin(c, sc)
        c.set_open_water(True, 1.0, 0.035, 0.06)
        c.set_surface_diffusion(0.024)
    v0 = dev.ledger()
    for _ in range(60):
        dev.step(DT, want_spray=False)
        ref.step(DT)
    for name in ("water", "slurry"):
        d = float(np.abs(dev.get(name) - ref.get(name)).max())
        assert d <= 1e-4, (name, d)
    du = float(np.abs(dev.get("uw") - ref.get("uw")).max())
    assert du <= 1e-3, du
    led = dev.ledger()
    gap = abs(led["total_m3"] + led["cut_m3"] - v0["total_m3"] - v0["cut_m3"]) / v0["total_m3"]
    assert gap < 1e-6, gap
    # The current slowed under the bed friction, as on the oracle.
    assert float(np.abs(dev.get("uw")).max()) < 0.9


def test_sample_reads_the_coarse_cell():
    sc = S.basin()
    dev = G.Sheet(res=sc["res"], cell=sc["cell"])
    ref = O.Core(threads=1)
    for c in (dev, ref):
        S.seed_basin(c, sc)
    for _ in range(5):
        dev.step(DT, want_spray=False)
        ref.step(DT)
    for x, z in ((0.3, -1.1), (2.0, 2.5), (-5.9, 0.1)):
        g = dev.sample(x, z)
        r = ref.sample(x, z)
        assert abs(g["water_m"] - r["water_m"]) <= 1e-4 and abs(g["bed_m"] - r["bed_m"]) == 0.0
        assert abs(g["moisture"] - r["moisture"]) == 0.0
    assert dev.sample(1000.0, 0.0) is None


def _pair_planes(ref, dev, names=("water", "slurry", "uw", "vw", "us", "vs", "moisture")):
    return {k: float(np.abs(ref.get(k) - dev.get(k)).max()) for k in names}


def test_recenter_scroll_and_jump_match_oracle():
    """Window moves between steps: a whole-cell scroll, a jump with no overlap
    (every cell parked), the way back; depths within the 1e-4 m criterion of
    the oracle throughout and the FP64 books (frozen included) equal."""
    scene = S.window200()
    ref, dev = O.Core(threads=1), G.Sheet()
    for c in (ref, dev):
        S.seed_core(c, scene)
    v0 = dev.ledger()["total_m3"]
    plan = [(3, None), (10, (3.1, -2.2)), (2, (100.0, 37.0)), (10, (0.0, 0.0)), (5, (-1.4, 0.8))]
    for steps, move in plan:
        if move is not None:
            ref.recenter(*move)
            dev.recenter(*move)
            assert dev.origin() == ref.origin()
            d = _pair_planes(ref, dev)
            assert d["water"] <= 1e-4 and d["slurry"] <= 1e-4 and d["moisture"] == 0.0, d
        for _ in range(steps):
            ref.step(DT)
            dev.step(DT, want_spray=False)
        d = _pair_planes(ref, dev)
        assert d["water"] <= 1e-4 and d["slurry"] <= 1e-4, (move, d)
        lr, ld = ref.ledger(), dev.ledger()
        assert abs(ld["frozen_water_m3"] - lr["frozen_water_m3"]) <= 1e-6 + 1e-5 * lr["frozen_water_m3"]
        assert abs(ld["frozen_slurry_m3"] - lr["frozen_slurry_m3"]) <= 1e-6 + 1e-5 * lr["frozen_slurry_m3"]
    led = dev.ledger()
    assert abs(led["total_m3"] + led["cut_m3"] - v0) <= 1e-6 * v0


@pytest.mark.parametrize("engine", [G.ENGINE_WINDOW, G.ENGINE_GRID])
def test_patch_water_outside_the_window_is_parked_and_restored(engine):
    """Tires at the window's west edge: the per-tire patches reach past it, so
    their off-window water is parked under its coarse world cell
    (src/fluid_core.rs:8484-8487); moving the window west restores it. The
    near field is off on both sides (the device releases tiles that leave the
    window; the reference keeps them by world cell)."""
    scene = S.grid(res=128, seed=0xABC, puddles=6)
    ox = S.snap_origin(0.0, 0.0, 128 * 0.2, 0.2)[0]
    ref = O.Core(res=128, fine_res=64, layout=1, threads=1)
    dev = G.Sheet(res=128, fine_res=64, layout=G.FINE_PER_TIRE, engine=engine)
    for c in (ref, dev):
        S.seed_core(c, scene)
        c.set_near_field(False)
        c.pour_water(ox - 1.0, ox + 2.0, -3.0, 3.0, 0.05)
    v0 = dev.ledger()["total_m3"]
    for k in range(20):
        # The west tires 0.2 m inside the window's edge: their patches reach 0.44 m past it.
        for t in S.tires_at(k * DT, speed=3.0, center=(ox + 0.95, 0.0), z0=-1.2):
            ref.push_tire(**t)
            dev.push_tire(**t)
        ref.step(DT)
        dev.step(DT, want_spray=False)
    lr, ld = ref.ledger(), dev.ledger()
    assert lr["frozen_water_m3"] > 0.0
    assert abs(ld["frozen_water_m3"] - lr["frozen_water_m3"]) <= 1e-3 * lr["frozen_water_m3"]
    for c in (ref, dev):
        c.recenter(-3.0, 0.0)
    lr, ld = ref.ledger(), dev.ledger()
    assert abs(ld["frozen_water_m3"] - lr["frozen_water_m3"]) <= 1e-6 + 1e-3 * lr["frozen_water_m3"]
    d = _pair_planes(ref, dev, ("water", "slurry"))
    assert d["water"] <= 1e-4 and d["slurry"] <= 1e-4, d
    led = dev.ledger()
    assert abs(led["total_m3"] + led["cut_m3"] - led["opened_m3"] - v0) <= 1e-5 * v0


@pytest.mark.parametrize("engine", [G.ENGINE_WINDOW, G.ENGINE_GRID])
def test_river_reach_and_wave_maker_match_oracle(engine):
    """A river channel through the window with the reach's inlet and outlet
    (src/fluid_core.rs:7638-7745), a paddle strip (:7420-7480) and open water:
    depth within 1e-4 m of the oracle after 60 steps, the reach bank within
    f32 rounding of the oracle's, and the FP64 books closed (the bank is on
    the ledger)."""
    sc = S.channel()
    reach = dict(along_z=False, positive=True, cross0=-4.0, cross1=4.0, rows=4, inlet_eta=0.3, outlet_eta=0.28,
                 inlet_speed_m_s=0.75)
    wave = dict(x0=5.0, x1=7.0, z0=-3.0, z1=3.0, dir_x=1.0, dir_z=0.0, amplitude_m_s=0.3, period_s=0.5, ramp_s=0.2)
    dev = G.Sheet(res=sc["res"], cell=sc["cell"], engine=engine)
    ref = O.Core(threads=1)
    for c in (dev, ref):
        S.seed_basin(c, sc)
        c.set_open_water(True, 1.0, 0.035, 0.06)
        c.set_river_reach(reach)
        c.set_wave_maker(wave)
    v0 = dev.ledger()
    for _ in range(60):
        dev.step(DT, want_spray=False)
        ref.step(DT)
    d = _pair_planes(ref, dev, ("water", "uw", "vw"))
    assert d["water"] <= 1e-4 and d["uw"] <= 1e-3, d
    led = dev.ledger()
    assert led["reach_m3"] > 0.0
    assert abs(led["reach_m3"] - ref.reach_bank_m3()) <= 1e-4 * led["reach_m3"] + 1e-6
    gap = abs(led["total_m3"] + led["cut_m3"] - v0["total_m3"] - v0["cut_m3"]) / v0["total_m3"]
    assert gap < 1e-6, gap
