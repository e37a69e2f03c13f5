"""Open-water mode on the oracle (FluidCore::set_open_water,
set_surface_diffusion; src/fluid_core.rs:5284-5303, :7485-7636): the
restatement behaves as the reference's comments say it must. The reference
has no unit test of these drivers alone (its open-water tests need the
bodies module), so these pin the restatement by its stated properties."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "dirty-gen_b200"))

import oracle  # noqa: E402
import silt_scenes as S  # noqa: E402

DT = 1.0 / 120.0


def run(steps, open_water=None, diffusion=0.0, scene=None):
    sc = scene or S.basin()
    c = oracle.Core(threads=1)
    S.seed_basin(c, sc)
    if open_water is not None:
        c.set_open_water(True, *open_water)
    c.set_surface_diffusion(diffusion)
    for _ in range(steps):
        c.step(DT)
    return c, sc


def band_speed(c, sc, lo=0.0, hi=3.0):
    res = sc["res"]
    x, z = S.cell_centres(res, sc["cell"], sc["origin"])
    u = c.get("uw").reshape(res, res)
    w = c.get("water").reshape(res, res)
    m = (np.abs(z) >= lo) & (np.abs(z) < hi) & (np.abs(x) < 4.0) & (w > 0.01)
    return float(np.abs(u[m]).mean())


def test_manning_friction_slows_the_current_and_never_reverses_it():
    free, sc = run(30, open_water=(1.0, 0.0, 0.0))
    rough, _ = run(30, open_water=(1.0, 0.05, 0.0))
    assert band_speed(rough, sc) < 0.99 * band_speed(free, sc)  # g n^2 |u| / h^(4/3) ~ 0.09 /s here
    res = sc["res"]
    x, z = S.cell_centres(res, sc["cell"], sc["origin"])
    u = rough.get("uw").reshape(res, res)
    core = (np.abs(z) < 2.0) & (np.abs(x) < 3.0)
    assert float(u[core].min()) > 0.0  # implicit: a current slows, it does not turn back


def test_eddy_viscosity_spreads_the_current_across_the_band_edge():
    plain, sc = run(30, open_water=(1.0, 0.0, 0.0))
    eddy, _ = run(30, open_water=(1.0, 0.0, 0.5))
    assert band_speed(eddy, sc, 3.0, 3.6) > band_speed(plain, sc, 3.0, 3.6) + 1e-3


def test_open_water_mobility_lets_a_slope_run_faster():
    sc = S.basin(speed=0.0)
    res = sc["res"]
    x, _ = S.cell_centres(res, sc["cell"], sc["origin"])
    w = sc["water"].reshape(res, res)
    tilt = np.where(w > 0, w + np.float32(0.05) * np.clip(-x / np.float32(6.0), -1, 1), 0).astype(np.float32)
    sc = dict(sc, water=tilt.ravel())
    mud, _ = run(20, scene=sc)
    open_, _ = run(20, open_water=(1.0, 0.0, 0.0), scene=sc)
    assert float(np.abs(open_.get("uw")).max()) > 3.0 * float(np.abs(mud.get("uw")).max())


def test_surface_diffusion_keeps_the_volume_and_smooths_the_surface():
    sc = S.basin(speed=0.0)
    res = sc["res"]
    rng = np.random.default_rng(5)
    w = sc["water"].copy()
    wet = w > 0.05
    w[wet] += (rng.standard_normal(int(wet.sum())) * 0.01).astype(np.float32)
    sc = dict(sc, water=np.maximum(w, 0).astype(np.float32))
    c0, _ = run(0, scene=sc)
    v0 = c0.ledger()["water64"]
    still, _ = run(5, scene=sc)
    diff, _ = run(5, diffusion=0.05, scene=sc)
    assert abs(diff.ledger()["water64"] - v0) <= 1e-5 * v0

    def roughness(c):
        eta = (c.get("water") + sc["bed"]).reshape(res, res)
        m = wet.reshape(res, res)[1:-1, 1:-1]
        lap = eta[1:-1, 2:] + eta[1:-1, :-2] + eta[2:, 1:-1] + eta[:-2, 1:-1] - 4 * eta[1:-1, 1:-1]
        return float(np.abs(lap[m]).mean())

    assert roughness(diff) < 0.95 * roughness(still)
