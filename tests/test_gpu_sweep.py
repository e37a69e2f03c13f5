"""The grid engine's Gauss-Seidel confinement against the oracle's step pair.

The reference's FluidCore::step_pair runs each sheet's inner loops serially,
so its coarse cells confine vorticity in a raster-order Gauss-Seidel sweep
(force_gravity_open, src/fluid_core.rs:2234-2260). The grid engine solves
that sweep as a fixed point across tiles (SILT_CONFINE_SWEEP, the default)
and the oracle's default Core is that step pair, so these scenes compare the
two forms the reference actually runs: the 2048 x 2048 grid with its inflow
strip and four per-tire 64 x 64 patches (the benchmark scene), windows picked
from a 256-window batch, and the 200 x 200 window.

Tolerance (the pass criterion): max |dh| <= 1e-4 m per layer after 100 steps.
"""
import numpy as np
import pytest

import oracle as O
import silt_b200 as G
import silt_scenes as S

pytestmark = pytest.mark.gpu
DT = 1.0 / 120.0
TOL_H = 1.0e-4


def bits_equal(a, b):
    return np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_grid_engine_sweep_is_bit_exact_on_window200():
    scene = S.window200()
    ref = O.Core()
    dev = G.Sheet(engine=G.ENGINE_GRID)
    dev.set_step_timing(True)
    for c in (ref, dev):
        S.seed_core(c, scene)
    for _ in range(100):
        ref.step(DT)
        dev.step(DT, want_spray=False)
    for name in ("water", "slurry", "uw", "vw", "us", "vs"):
        a, b = ref.get(name), dev.get(name)
        assert bits_equal(a, b), (name, float(np.abs(a - b).max()))
    parts = dev.step_parts()
    print("sweep launches", parts["sweep_launches"], "most passes", parts["sweep_passes_max"],
          "fallbacks", parts["sweep_fallbacks"])
    assert parts["sweep_launches"] == 100 and parts["sweep_fallbacks"] == 0


def test_confinement_form_is_checked():
    dev = G.Sheet(res=64, engine=G.ENGINE_GRID)
    dev.set_confinement(G.CONFINE_SNAPSHOT)
    dev.set_confinement(G.CONFINE_SWEEP)
    with pytest.raises(G.SiltError):
        dev.set_confinement(7)


def test_grid2048_with_tire_patches_and_inflow_matches_step_pair():
    """The benchmark scene: 2048 x 2048 grid, eight puddles, the rut slurry,
    0.5 m^3/s inflow on row 0 and four tires at 5 m/s each with its own
    64 x 64 patch of 2 cm cells, 100 steps against the oracle's step pair."""
    scene = S.grid(res=2048)
    ref = O.Core(res=2048, fine_res=64, layout=1, threads=2)
    dev = G.Sheet(res=2048, fine_res=64, layout=G.FINE_PER_TIRE)
    for c in (ref, dev):
        S.seed_core(c, scene)
        c.set_inflow(0, -2.0, 2.0, 0.5)
    ev_r = ev_d = 0
    for k in range(100):
        for t in S.tires_at(k * DT, speed=5.0):
            ref.push_tire(**t)
            dev.push_tire(**t)
        ev_r += len(ref.step(DT))
        ev_d += len(dev.step(DT))
    out = {}
    for name in ("water", "slurry"):
        a, b = ref.get(name), dev.get(name)
        out[name] = (float(np.abs(a - b).max()), bool(bits_equal(a, b)))
    print("max |dh| and bit equality", out, "spray events", ev_r, ev_d)
    assert out["water"][0] <= TOL_H and out["slurry"][0] <= TOL_H, out
    lr, ld = ref.ledger(), dev.ledger()
    assert abs(ld["water_m3"] - lr["water64"]) <= 1e-6 * lr["water64"]
    assert abs(ld["slurry_m3"] - lr["slurry64"]) <= 1e-6 * lr["slurry64"]


def test_batch_windows_match_their_oracle_step_pairs():
    """From the 256-window batch (sides log-uniform 64..512, 1..4 puddles,
    0..4 tires with 64 x 64 patches), ten windows spanning the sizes, with
    and without tires, each against its own oracle step pair after 100 batch
    steps."""
    wins = S.batch_windows(n=256)
    order = sorted(range(len(wins)), key=lambda w: wins[w]["res"])
    picked = []
    for q in np.linspace(0, len(order) - 1, 8).astype(int):
        picked.append(order[q])
    for want_tires in (True, False):  # make sure both kinds are in
        if not any((wins[w]["tires"] > 0) == want_tires for w in picked):
            picked.append(next(w for w in order[::-1] if (wins[w]["tires"] > 0) == want_tires))
    picked = sorted(set(picked))
    import torch

    stream = torch.cuda.Stream()
    sheets = []
    for w in wins:
        sh = G.Sheet(res=w["res"], fine_res=64, layout=G.FINE_PER_TIRE, engine=G.ENGINE_GRID,
                     stream=stream.cuda_stream)
        S.seed_core(sh, w)
        sheets.append(sh)
    batch = G.Batch(sheets)
    refs = {}
    for w in picked:
        refs[w] = O.Core(res=wins[w]["res"], fine_res=64, layout=1)
        S.seed_core(refs[w], wins[w])

    def tires(k, win):
        if not win["tires"]:
            return []
        return S.tires_at(k * DT, speed=5.0, z0=-0.5 * win["res"] * 0.2)[:win["tires"]]

    for k in range(1, 101):
        idx, ts = [], []
        for w, win in enumerate(wins):
            for t in tires(k, win):
                idx.append(w)
                ts.append(t)
                if w in refs:
                    refs[w].push_tire(**t)
        batch.push_tires(idx, ts)
        batch.step(DT)
        for w in picked:
            refs[w].step(DT)
    worst = {}
    for w in picked:
        d = {name: float(np.abs(refs[w].get(name) - sheets[w].get(name)).max()) for name in ("water", "slurry")}
        worst[(wins[w]["res"], wins[w]["tires"])] = d
        assert d["water"] <= TOL_H and d["slurry"] <= TOL_H, (w, wins[w]["res"], wins[w]["tires"], d)
    print("picked windows (side, tires) -> max |dh|", worst)
    sizes = [wins[w]["res"] for w in picked]
    assert min(sizes) < 80 and max(sizes) > 400
    batch.close()
