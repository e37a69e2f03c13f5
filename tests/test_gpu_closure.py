"""The learned closure inside the step: coupling modes, the network input,
volume bookkeeping of the correction, the fallback to the nested sheets, and
the batched form against the single-window form."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import silt_b200 as G
import silt_closure as C
import silt_closure_train as T
import silt_scenes as S

pytestmark = pytest.mark.gpu

DT = 1.0 / 120.0


def sheet(sc, stream=None, engine=G.ENGINE_GRID):
    sh = G.Sheet(res=T.RES, cell=T.CELL, fine_res=T.FINE_RES, fine_cell=0.02, layout=G.FINE_PER_TIRE,
                 stream=stream, engine=engine)
    S.seed_core(sh, sc)
    return sh


def ident_norm():
    n = np.zeros(C.NNORM, np.float32)
    n[6:12] = 1.0
    n[12:20] = 1.0
    return n


def strong_params(seed=2, gain=4.0):
    """An untrained network scaled up so its corrections are visible."""
    p = torch.tensor(C.init_params(seed))
    P = C.split_params(p)  # views into p
    P["W3"].mul_(gain)
    P["b3"][:C.OUT_USED] = 0.01
    return p.numpy()


def step_with(sh, sc, step):
    for t in T.scene_tires(sc, step):
        sh.push_tire(**t)
    sh.step(DT, want_spray=False)


def test_none_coupling_lays_no_patch_and_conserves():
    sc = T.drive_scene(1)
    a, b = sheet(sc), sheet(sc)
    C.set_coupling(b, C.COUPLING_NONE)
    v0 = a.ledger()["total_m3"]
    for step in range(1, 31):
        step_with(a, sc, step)
        step_with(b, sc, step)
    la, lb = a.ledger(), b.ledger()
    # The books close to what the dry cut removes (films under 1e-6 m,
    # src/fluid_core.rs:2072-2081): a few 1e-6 of the volume per step here.
    assert abs(lb["total_m3"] - v0) <= 2e-4 * v0, (lb, v0)
    assert abs(la["total_m3"] - v0) <= 2e-4 * v0, (la, v0)
    diff = np.abs(a.get("water") - b.get("water")).max()
    assert diff > 0.0  # the nested sheets change the flow near the tires


def test_features_are_the_raw_state_around_the_vehicle():
    sc = T.drive_scene(2)
    sh = sheet(sc)
    for step in range(1, 6):
        step_with(sh, sc, step)
    probe = C.Closure(np.zeros(C.NPARAM, np.float32), ident_norm())
    tires = T.scene_tires(sc, 6)
    for t in tires:
        sh.push_tire(**t)
    x = torch.zeros((1, C.CROP, C.CROP, C.CIN), dtype=torch.bfloat16, device="cuda")
    ci0, cj0 = C.features(sh, probe, x)
    torch.cuda.synchronize()
    mx = np.mean([t["x"] for t in tires], dtype=np.float32)
    mz = np.mean([t["z"] for t in tires], dtype=np.float32)
    ox, oz = S.snap_origin(0.0, 0.0, T.RES * T.CELL, T.CELL)
    assert ci0 == int(np.floor((mx - ox) / T.CELL)) - 16 and cj0 == int(np.floor((mz - oz) / T.CELL)) - 16
    res = T.RES
    planes = {k: sh.get(k).reshape(res, res) for k in ("water", "slurry", "uw", "vw", "bed")}
    xs = x[0].float().cpu().numpy()
    for cy in range(0, C.CROP, 3):
        for cx in range(0, C.CROP, 3):
            i, j = ci0 + cx, cj0 + cy
            hw = planes["water"][j, i]
            want = [hw, planes["slurry"][j, i], planes["uw"][j, i] if hw >= 1e-6 else 0.0,
                    planes["vw"][j, i] if hw >= 1e-6 else 0.0, planes["bed"][j, i]]
            for c, v in enumerate(want):
                assert abs(xs[cy, cx, c] - v) <= 2.0 ** -8 * abs(v) + 1e-30, (cx, cy, c, xs[cy, cx, c], v)
            assert np.all(xs[cy, cx, C.IN_USED:] == 0.0)
    shove = xs[:, :, 5]
    assert shove.max() >= 0.4 and shove.min() == 0.0  # the tires' footprints are in the crop
    probe.close()
    sh.close()


def test_closure_correction_is_volume_neutral_and_booked():
    sc = T.drive_scene(3)
    net = C.Closure(strong_params(), ident_norm() * np.r_[np.ones(12), np.full(8, 1e-3)].astype(np.float32))
    sh = sheet(sc)
    C.set_coupling(sh, C.COUPLING_CLOSURE, net, threshold=1e9)
    v0 = sh.ledger()["total_m3"]
    for step in range(1, 41):
        step_with(sh, sc, step)
        led = sh.ledger()
        for name, key in (("water", "water_m3"), ("slurry", "slurry_m3")):
            h = sh.get(name).astype(np.float64)
            assert np.all(h >= 0.0) and np.all(np.isfinite(h))
            area = float(np.float32(T.CELL)) ** 2  # the sheet's f32 cell size
            assert abs(h.sum() * area - led[key]) <= 1e-9 * max(led[key], 1e-12), (step, key)
    st = C.stats(sh)
    assert st["closure_steps"] == 40 and st["fallback_steps"] == 0 and st["moved_m3"] > 0.0
    assert abs(sh.ledger()["total_m3"] - v0) <= 2e-4 * v0
    sh.close()
    net.close()


def test_residual_above_threshold_falls_back_to_the_nested_sheets():
    sc = T.drive_scene(4)
    # Outputs far larger than any depth: the limiter clips most of every transfer.
    net = C.Closure(strong_params(gain=50.0), ident_norm())
    sh = sheet(sc)
    C.set_coupling(sh, C.COUPLING_CLOSURE, net, threshold=0.05)
    for step in range(1, 21):
        step_with(sh, sc, step)
    st = C.stats(sh)
    assert st["closure_steps"] > 0 and st["fallback_steps"] > 0, st
    assert st["closure_steps"] + st["fallback_steps"] == 20
    assert st["last_residual"] > 0.05
    sh.close()
    net.close()


def test_batched_closure_matches_single_windows():
    scenes = [T.drive_scene(10 + k) for k in range(3)]
    keep = torch.cuda.Stream()  # one stream for every sheet of the batch
    stream = keep.cuda_stream
    net = C.Closure(strong_params(), ident_norm() * np.r_[np.ones(12), np.full(8, 1e-3)].astype(np.float32))
    alone = [sheet(sc, stream) for sc in scenes]
    grouped = [sheet(sc, stream) for sc in scenes]
    modes = (C.COUPLING_CLOSURE, C.COUPLING_NONE, C.COUPLING_CLOSURE)
    for sh_a, sh_b, m in zip(alone, grouped, modes):
        C.set_coupling(sh_a, m, net if m == C.COUPLING_CLOSURE else None, 1e9)
        C.set_coupling(sh_b, m, net if m == C.COUPLING_CLOSURE else None, 1e9)
    batch = G.Batch(grouped)
    for step in range(1, 16):
        idx, recs = [], []
        for k, sc in enumerate(scenes):
            for t in T.scene_tires(sc, step):
                alone[k].push_tire(**t)
                idx.append(k)
                recs.append(t)
            alone[k].step(DT, want_spray=False)
        batch.push_tires(idx, recs)
        batch.step(DT)
    for k in range(len(scenes)):
        for name in ("water", "slurry", "uw", "vw", "us", "vs"):
            a, b = alone[k].get(name), grouped[k].get(name)
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (k, name, float(np.abs(a - b).max()))
    batch.close()
    net.close()


def test_pairs_and_training_on_a_small_set():
    xs, ts, wins, stp = T.generate(n_windows=4, steps=12, log=lambda *a: None)
    assert tuple(xs.shape) == (48, C.CROP, C.CROP, C.CIN) and tuple(ts.shape) == (48, C.CROP, C.CROP, 8)
    assert float(ts[..., :2].abs().max()) > 0.0  # the nested sheets moved water the tire-less coarse step did not
    assert float(ts[..., :2].sum(dim=(1, 2)).abs().max()) < 1e-4  # mean removed: what face transfers can carry
    assert float(ts[..., 2:6].abs().max()) > 0.0 and set(torch.unique(ts[..., 6:]).tolist()) <= {0.0, 1.0}
    held = (wins >= 3).to("cuda")
    norm = T.norm_block(xs[~held], ts[~held])
    assert norm.shape == (C.NNORM,) and np.all(np.isfinite(norm))
    assert np.all(norm[6:12] > 0) and np.all(norm[12:] > 0)
    params, report = T.train(xs, ts, norm, held, epochs=40, batch=32, log=lambda *a: None)
    assert params.shape == (C.NPARAM,) and np.all(np.isfinite(params))
    first, last = report["history"][0][1], report["history"][-1][1]
    assert last < first, report["history"]
    assert report["train"]["water_depth_change_rel_l2"] < 1.0


def test_step_loss_gradient_matches_autograd():
    n = 3
    g = torch.Generator(device="cuda").manual_seed(5)
    y = torch.randn((n, C.CROP, C.CROP, C.COUT), device="cuda", generator=g)
    t = torch.randn((n, C.CROP, C.CROP, 8), device="cuda", generator=g) * 1e-3
    t[..., 6:] = (torch.rand((n, C.CROP, C.CROP, 2), device="cuda", generator=g) > 0.3).float()
    scale = torch.tensor([1e-3, 2e-3, 5e-4, 7e-4, 0.1, 0.2, 0.05, 0.07], device="cuda")
    inv_var = torch.tensor([1e6, 4e6, 100.0, 25.0, 400.0, 200.0], device="cuda")
    lam = 0.01
    dy, loss = C.step_loss_grad(y, t, scale, inv_var, lam)
    yr = y.clone().requires_grad_(True)
    G = yr[..., :8] * scale
    mask = torch.ones_like(G)
    mask[:, :, -1, 0:4:2] = 0.0
    mask[:, -1, :, 1:4:2] = 0.0
    G = G * mask
    total = 0.0
    for l in range(2):
        d = T.divergence(G[..., 2 * l], G[..., 2 * l + 1])
        total = total + (inv_var[l] * (d - t[..., l]) ** 2).sum()
        for k in (2 * l, 2 * l + 1):
            total = total + (inv_var[2 + k] * t[..., 6 + l] * (G[..., 4 + k] - t[..., 2 + k]) ** 2).sum()
    total = total + lam * (yr[..., :8] ** 2).sum()
    total = total / (n * C.CROP * C.CROP)
    total.backward()
    ref_loss = float(total.detach())
    assert abs(float(loss) - ref_loss) <= 1e-4 * ref_loss
    ref = yr.grad
    err = float((dy.float() - ref).abs().max()) / float(ref.abs().max())
    assert err < 2.0 ** -7, err
