"""Training of the learned flux closure on pairs the nested 2 cm sheets make.

Data (the closure training-set recipe): windows of 200 x 200 coarse cells
(20 cm) built like the reference's 200-cell test window (bed noise, rut pair,
puddle, slurry in the ruts), each with its own seed, driven by one vehicle of
four tires at a speed drawn from U(2, 10) m/s along the ruts. Every step of
every window gives one pair: the state before the step, and the depth the
nested 2 cm sheets (64 x 64 per tire) leave after it minus the depth the
closure's own coarse step (no sheets, no tire shove) leaves from the same
state, on the 32 x 32 crop around the vehicle, per layer, less its mean (the
part face transfers can carry). The network predicts face transfers; the loss
is the error of the depth change they make (their divergence), so the
network is free to choose local transfers.

Run as a script on a GPU: it generates the pairs, trains with the library's
tensor-core kernels and Adam, reports train and held-out errors, and writes
the parameters and normalisation block (`--out`, numpy .npz).
"""
import argparse
import json
import math
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
    sys.path.insert(0, HERE)

import silt_b200  # noqa: E402
import silt_closure as C  # noqa: E402
import silt_scenes as S  # noqa: E402

DT = 1.0 / 120.0
CELL = 0.2
RES = 200
FINE_RES = 64


def drive_scene(k, base_seed=0x5EED0C10):
    """Window k: the 200-cell test window with seed base_seed + k and one
    vehicle (1.5 m track, 2.4 m wheelbase) on the ruts, speed U(2, 10) m/s,
    starting z U(-5, 1) m, lateral offset U(-0.3, 0.3) m, load U(3, 5) kN
    (recorded; the sheet's tire shove has no load term)."""
    rng = np.random.default_rng(base_seed + 7919 * k)
    sc = S.window200(seed=base_seed + k, res=RES, cell=CELL)
    sc["speed"] = float(rng.uniform(2.0, 10.0))
    sc["z0"] = float(rng.uniform(-5.0, 1.0))
    sc["x0"] = float(rng.uniform(-0.3, 0.3))
    sc["load_kn"] = float(rng.uniform(3.0, 5.0))
    return sc


def scene_tires(sc, step):
    return S.tires_at(step * DT, speed=sc["speed"], center=(sc["x0"], 0.0), z0=sc["z0"])


def make_sheets(scenes, stream, mode=C.COUPLING_NESTED, net=None, threshold=0.25):
    out = []
    for sc in scenes:
        sh = silt_b200.Sheet(res=RES, cell=CELL, fine_res=FINE_RES, fine_cell=0.02, layout=silt_b200.FINE_PER_TIRE,
                             device=0, stream=stream, engine=silt_b200.ENGINE_GRID)
        S.seed_core(sh, sc)
        if mode != C.COUPLING_NESTED:
            C.set_coupling(sh, mode, net, threshold)
        out.append(sh)
    return out


def push_all(batch, scenes, step):
    idx, recs = [], []
    for k, sc in enumerate(scenes):
        for t in scene_tires(sc, step):
            idx.append(k)
            recs.append(t)
    batch.push_tires(idx, recs)


def divergence(gx, gz):
    """Depth change of each cell from face transfers (the step's correction rule)."""
    import torch

    inflow = torch.zeros_like(gx)
    inflow[..., :, 1:] += gx[..., :, :-1]
    inflow[..., 1:, :] += gz[..., :-1, :]
    return inflow - gx - gz


def crop(plane, ci0, cj0):
    """plane [res, res] (rows j) -> [32, 32] crop at (ci0, cj0), zero outside."""
    import torch

    n = C.CROP
    out = torch.zeros((n, n), dtype=plane.dtype, device=plane.device)
    res = plane.shape[0]
    i0, j0 = max(ci0, 0), max(cj0, 0)
    i1, j1 = min(ci0 + n, res), min(cj0 + n, res)
    if i0 < i1 and j0 < j1:
        out[j0 - cj0:j1 - cj0, i0 - ci0:i1 - ci0] = plane[j0:j1, i0:i1]
    return out


def generate(n_windows=128, steps=160, base_seed=0x5EED0C10, log=print, rollout=None):
    """Pairs from n_windows x steps steps. The states come from the nested run
    itself, or with `rollout` = (params, norm) from windows the closure with
    that network drives (each step's state copied into a nested and a
    coarse-only window for the target), so the network also learns from the
    states its own corrections lead to. Returns (x_raw [N, 32, 32, 16] BF16
    raw inputs, targets [N, 32, 32, 8] FP32: water and slurry depth change
    (m, mean removed), water u, v and slurry u, v change (m/s, where the
    coarse step left the cell wet), water and slurry wet weights; window index
    [N], step [N])."""
    import torch

    st = torch.cuda.Stream()  # the sheets, batches and crop arithmetic share one stream
    with torch.cuda.stream(st):
        out = _generate(n_windows, steps, base_seed, st.cuda_stream, log, rollout)
    torch.cuda.synchronize()
    return out


def _generate(n_windows, steps, base_seed, stream, log, rollout):
    import torch

    scenes = [drive_scene(k, base_seed) for k in range(n_windows)]
    ident = np.zeros(C.NNORM, np.float32)
    ident[6:12] = 1.0
    ident[12:20] = 1.0
    probe = C.Closure(np.zeros(C.NPARAM, np.float32), ident)  # raw inputs, no correction
    nested = make_sheets(scenes, stream)
    plain = make_sheets(scenes, stream, C.COUPLING_CLOSURE, probe, 1e30)
    bn, bp = silt_b200.Batch(nested), silt_b200.Batch(plain)
    drive_net, driven, bd = None, None, None
    if rollout is not None:
        drive_net = C.Closure(rollout[0], rollout[1])
        driven = make_sheets(scenes, stream, C.COUPLING_CLOSURE, drive_net, 1e30)
        bd = silt_b200.Batch(driven)
    src = driven if driven is not None else nested
    N = n_windows * steps
    xs = torch.zeros((N, C.CROP, C.CROP, C.CIN), dtype=torch.bfloat16, device="cuda")
    dhs = torch.zeros((N, C.CROP, C.CROP, 8), dtype=torch.float32, device="cuda")
    wins = torch.zeros(N, dtype=torch.int32)
    stp = torch.zeros(N, dtype=torch.int32)
    t0 = time.time()
    q = 0
    for step in range(1, steps + 1):
        for k in range(n_windows):
            plain[k].copy_state_from(src[k])
            if driven is not None:
                nested[k].copy_state_from(src[k])
        push_all(bn, scenes, step)
        origins = []
        for k in range(n_windows):
            origins.append(C.features(nested[k], probe, xs[q + k:q + k + 1]))
        push_all(bp, scenes, step)
        bn.step(DT)
        bp.step(DT)
        if bd is not None:
            push_all(bd, scenes, step)
            bd.step(DT)
        t = torch.zeros((n_windows, 8, C.CROP, C.CROP), dtype=torch.float32, device="cuda")
        for k in range(n_windows):
            ci0, cj0 = origins[k]
            for l, (hn, un, vn) in enumerate((("water", "uw", "vw"), ("slurry", "us", "vs"))):
                hb = crop(plain[k].plane_device(hn), ci0, cj0)
                t[k, l] = crop(nested[k].plane_device(hn), ci0, cj0) - hb
                wet = (hb >= 1e-6).float()
                for m, name in ((0, un), (1, vn)):
                    t[k, 2 + 2 * l + m] = (crop(nested[k].plane_device(name), ci0, cj0) -
                                           crop(plain[k].plane_device(name), ci0, cj0)) * wet
                t[k, 6 + l] = wet
            wins[q + k] = k
            stp[q + k] = step
        t[:, :2] -= t[:, :2].mean(dim=(-2, -1), keepdim=True)
        dhs[q:q + n_windows] = t.permute(0, 2, 3, 1)
        q += n_windows
        if step % 40 == 0:
            log(f"generate: step {step}/{steps}, {time.time() - t0:.1f} s")
    for b in (bn, bp, bd):
        if b is not None:
            b.close()
    for sh in nested + plain + (driven or []):
        sh.close()
    probe.close()
    if drive_net is not None:
        drive_net.close()
    return xs, dhs, wins, stp


def norm_block(xs, dhs):
    """Input means and inverse deviations, and the output scales: each
    layer's transfers in units of its depth-change deviation, each velocity
    change in units of its deviation over wet cells."""
    import torch

    x = xs[..., :C.IN_USED].float().reshape(-1, C.IN_USED)
    mean = x.mean(0)
    std = x.std(0).clamp_min(1e-6)
    t = dhs.reshape(-1, 8)
    sd = t[:, :2].std(0).clamp_min(1e-9)
    sv = []
    for k in range(4):
        w = t[:, 6 + k // 2]
        sv.append(torch.sqrt((t[:, 2 + k] ** 2 * w).sum() / w.sum().clamp_min(1.0)).clamp_min(1e-6))
    scale = torch.stack([sd[0], sd[0], sd[1], sd[1]] + sv)
    return torch.cat([mean, 1.0 / std, scale]).cpu().numpy().astype(np.float32)


def normalise(xs, norm):
    import torch

    n = torch.tensor(norm, device=xs.device)
    x = xs.float()
    x[..., :C.IN_USED] = (x[..., :C.IN_USED] - n[:C.IN_USED]) * n[6:12]
    return x.to(torch.bfloat16)


def train(xs, dhs, norm, held, epochs=20, batch=256, lr=2e-3, lam=1e-3, seed=0, log=print):
    """Adam on the step loss (each layer's depth-change error and each
    velocity-change error over its deviation, squared) plus lam times the
    squared network outputs (a preference for small corrections). Returns
    (params, report)."""
    import torch

    xn = normalise(xs, norm)
    scale = torch.tensor(norm[12:20], device=xs.device)
    inv_var = 1.0 / torch.stack([scale[0], scale[2], scale[4], scale[5], scale[6], scale[7]]) ** 2
    train_idx = torch.nonzero(~held).flatten()
    held_idx = torch.nonzero(held).flatten()
    net = C.Net(C.init_params(seed))
    opt = C.Adam(net, lr=lr)
    gen = torch.Generator(device="cpu").manual_seed(seed)
    iters = max(1, epochs * len(train_idx) // batch)
    t0 = time.time()
    history = []
    for it in range(iters):
        sel = train_idx[torch.randint(len(train_idx), (batch,), generator=gen)].to(xs.device)
        x = xn[sel].contiguous()
        a1, a2, y = net.forward(x)
        dy, loss = C.step_loss_grad(y, dhs[sel].contiguous(), scale, inv_var, lam)
        g = net.grads(x, a1, a2, dy)
        frac = it / iters
        opt.step(g, lr=lr * 0.5 * (1.0 + math.cos(math.pi * frac)))
        if it % 200 == 0 or it == iters - 1:
            history.append((it, float(loss)))
            log(f"train: iter {it}/{iters} loss {float(loss):.5f} ({time.time() - t0:.1f} s)")
    report = {"iters": iters, "history": history, "seconds": time.time() - t0, "lambda": lam}
    report["train"] = evaluate(net, xn, dhs, scale, train_idx[:2048])
    report["held_out"] = evaluate(net, xn, dhs, scale, held_idx)
    return net.p.detach().cpu().numpy(), report


def evaluate(net, xn, dhs, scale, idx, chunk=512):
    """Relative L2 errors of the depth change the predicted transfers make and
    of the predicted velocity change (wet cells), per layer (predicting no
    change scores 1)."""
    import torch

    num = [0.0] * 4
    den = [0.0] * 4
    for s in range(0, len(idx), chunk):
        sel = idx[s:s + chunk].to(xn.device)
        _, _, y = net.forward(xn[sel].contiguous())
        g = y[..., :C.OUT_USED] * scale
        g[:, :, -1, 0:4:2] = 0.0  # no transfer across the crop's edge: x faces of the last column,
        g[:, -1, :, 1:4:2] = 0.0  # z faces of the last row
        t = dhs[sel]
        for l in range(2):
            d = divergence(g[..., 2 * l], g[..., 2 * l + 1])
            num[l] += float(((d - t[..., l]) ** 2).sum())
            den[l] += float((t[..., l] ** 2).sum())
            w = t[..., 6 + l]
            for k in (2 * l, 2 * l + 1):
                num[2 + l] += float((((g[..., 4 + k] - t[..., 2 + k]) ** 2) * w).sum())
                den[2 + l] += float(((t[..., 2 + k] ** 2) * w).sum())
    r = [math.sqrt(a / max(b, 1e-30)) for a, b in zip(num, den)]
    return {"water_depth_change_rel_l2": r[0], "slurry_depth_change_rel_l2": r[1],
            "water_velocity_change_rel_l2": r[2], "slurry_velocity_change_rel_l2": r[3], "pairs": int(len(idx))}


def main(argv=None):
    import torch

    ap = argparse.ArgumentParser()
    ap.add_argument("--windows", type=int, default=128)
    ap.add_argument("--steps", type=int, default=160)
    ap.add_argument("--epochs", type=int, default=60)
    ap.add_argument("--held-windows", type=int, default=13)
    ap.add_argument("--rollouts", type=int, default=1, help="rounds of pairs from closure-driven windows")
    ap.add_argument("--out", default=os.path.join(HERE, "closure_weights.npz"))
    ap.add_argument("--report", default=None)
    a = ap.parse_args(argv)
    torch.cuda.set_device(0)
    xs, dhs, wins, _ = generate(a.windows, a.steps)
    held = (wins >= a.windows - a.held_windows).to("cuda")
    norm = norm_block(xs[~held], dhs[~held])
    params, report = train(xs, dhs, norm, held, epochs=a.epochs)
    rounds = [report]
    # Rollout rounds: states the closure's own corrections lead to, targets
    # from the nested and coarse-only steps of copies of them.
    for r in range(a.rollouts):
        xr, dr, wr, _ = generate(a.windows, a.steps, rollout=(params, norm))
        xs, dhs = torch.cat([xs, xr]), torch.cat([dhs, dr])
        wins = torch.cat([wins, wr])
        held = (wins >= a.windows - a.held_windows).to("cuda")
        params, report = train(xs, dhs, norm, held, epochs=max(1, a.epochs // (r + 2)))
        rounds.append(report)
    report = dict(report)
    report["rounds"] = [{k: v for k, v in rr.items() if k != "history"} for rr in rounds]
    report.update({"windows": a.windows, "steps": a.steps, "pairs": int(xs.shape[0]),
                   "held_windows": a.held_windows, "rollouts": a.rollouts, "norm": norm.tolist()})
    np.savez(a.out, params=params.astype(np.float32), norm=norm)
    print(json.dumps({k: v for k, v in report.items() if k != "history"}), flush=True)
    if a.report:
        with open(a.report, "w") as f:
            json.dump(report, f, indent=1)


if __name__ == "__main__":
    main()
