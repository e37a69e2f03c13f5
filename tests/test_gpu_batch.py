"""Batched windows: silt_batch_step must give every window exactly what
silt_step gives it alone (the same kernels and arithmetic; only the FP64
ledger sums may differ in their last bits, from the order of the atomics)."""
import numpy as np
import pytest

import silt_b200 as G
import silt_shard
import silt_scenes as S

pytestmark = pytest.mark.gpu
DT = 1.0 / 120.0


def make(scene, fast=False, stream=None):
    sh = G.Sheet(res=scene["res"], cell=0.2, fine_res=64, fine_cell=0.02, layout=G.FINE_PER_TIRE,
                 engine=G.ENGINE_GRID, stream=stream)
    S.seed_core(sh, scene)
    if fast:
        n = scene["res"] ** 2
        sh.map_water_velocity(np.full(n, 14.0, np.float32), np.full(n, -3.0, np.float32))
    return sh


def push(sh, k, count):
    for t in S.tires_at(k * DT, speed=5.0, z0=-3.0)[:count]:
        sh.push_tire(**t)


def test_batch_step_equals_single_steps():
    scenes = [S.grid(res=r, seed=0x1234 + r, puddles=3) for r in (64, 96, 130, 200)]
    opts = [dict(), dict(fast=True), dict(tires=True), dict(tires=True, fast=True)]
    import torch

    stream = torch.cuda.Stream()
    alone = [make(sc, o.get("fast", False)) for sc, o in zip(scenes, opts)]
    grouped = [make(sc, o.get("fast", False), stream.cuda_stream) for sc, o in zip(scenes, opts)]
    batch = G.Batch(grouped)
    for k in range(1, 25):
        idx, tires = [], []
        for w, o in enumerate(opts):
            if o.get("tires"):
                push(alone[w], k, 2 + w % 3)
                for t in S.tires_at(k * DT, speed=5.0, z0=-3.0)[:2 + w % 3]:
                    idx.append(w)
                    tires.append(t)
            alone[w].step(DT, want_spray=False)
        batch.push_tires(idx, tires)  # the batch's bulk form of push_tire
        batch.step(DT)
    for w in range(len(scenes)):
        for name in ("water", "slurry", "uw", "vw", "us", "vs"):
            a, b = alone[w].get(name), grouped[w].get(name)
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (w, name, float(np.abs(a - b).max()))
        la, lb = alone[w].ledger(), grouped[w].ledger()
        for key in ("water_m3", "slurry_m3", "spray_m3"):
            assert abs(la[key] - lb[key]) <= 1e-12 * max(1.0, abs(la[key])), (w, key)
    gathered = batch.ledgers()
    for w in range(len(scenes)):
        single = grouped[w].ledger()
        for key in ("water_m3", "slurry_m3", "spray_m3", "frozen_water_m3", "opened_m3", "total_m3"):
            assert gathered[w][key] == single[key], (w, key)
    rows = batch.ledger_rows()
    for w in range(len(scenes)):
        assert list(rows[w]) == [gathered[w][k] for k in silt_shard.LEDGER_KEYS], w
    parts = batch.parts()
    assert parts["steps"] == 24 and parts["launches"] > 0
    batch.close()


def test_batch_refuses_window_engine_sheets_and_mixed_streams():
    sh = G.Sheet(res=64, engine=G.ENGINE_WINDOW)
    with pytest.raises(G.SiltError):
        G.Batch([sh])
    a, b = G.Sheet(res=64, engine=G.ENGINE_GRID), G.Sheet(res=64, engine=G.ENGINE_GRID)
    with pytest.raises(G.SiltError, match="one stream"):
        G.Batch([a, b])


def _batch_of(scenes, stream):
    sheets = [make(sc, False, stream.cuda_stream) for sc in scenes]
    return sheets, G.Batch(sheets)


def _drive(batch, n_win, steps):
    for k in range(1, steps + 1):
        idx, tires = [], []
        for w in range(n_win):
            for t in S.tires_at(k * DT, speed=5.0, z0=-3.0)[:1 + w % 3]:
                idx.append(w)
                tires.append(t)
        batch.push_tires(idx, tires)
        batch.step(DT)


def test_batch_autotuner_times_real_steps_and_changes_no_bit():
    """The autotuner (silt_batch_autotune) picks the batched sweep's CTAs per
    SM, the transport's grid and the tracer passes' blocks by timing the
    batch's own steps; every candidate computes the same bits, so a tuned
    batch, one with explicit settings and one on the defaults end equal. A
    second batch of the same size class takes the kept choice without trials."""
    import torch

    scenes = [S.grid(res=r, seed=0x77 + r, puddles=3) for r in (64, 100, 160)]
    stream = torch.cuda.Stream()
    runs = {}
    for mode in ("default", "tuned", "set"):
        sheets, b = _batch_of(scenes, stream)
        if mode == "tuned":
            b.autotune(True)
        elif mode == "set":
            b.set_tune(sweep_ctas_per_sm=1, transport_blocks=296, tracer_blocks=1184)
        _drive(b, len(scenes), 26)  # six untimed steps, then 8 candidates x 2 timed steps
        runs[mode] = (sheets, b, b.tune())
    t = runs["tuned"][2]
    assert t["tuned"] and t["trials"] == 8 and all(x > 0.0 for x in t["trial_ms"]), t
    assert t["sweep_ctas_per_sm"] in (1, 2) and t["transport_blocks"] in (296, 592, 1184)
    assert t["tracer_blocks"] in (1184, 2368, 4736)
    assert runs["set"][2]["sweep_ctas_per_sm"] == 1 and not runs["set"][2]["tuned"]
    for mode in ("tuned", "set"):
        for w in range(len(scenes)):
            for name in ("water", "slurry", "uw", "vw", "foam", "turbid", "susp"):
                a, c = runs["default"][0][w].get(name), runs[mode][0][w].get(name)
                assert np.array_equal(a.view(np.uint32), c.view(np.uint32)), (mode, w, name)
    sheets, b = _batch_of(scenes, stream)
    b.autotune(True)
    again = b.tune()
    assert again["tuned"] and again["trials"] == 0
    for k in ("sweep_ctas_per_sm", "transport_blocks", "tracer_blocks"):
        assert again[k] == t[k]
    b.close()
    for _, bb, _ in runs.values():
        bb.close()
