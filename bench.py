"""Benchmark of the B200 two-layer sheet step.

Workload (one "step" = one FluidCore-style step of the whole grid): a
2048 x 2048 grid of 0.2 m cells, seeded 4-octave value-noise bed, eight
seeded puddles 0.05-0.2 m deep and 2-8 m across, a clay slurry rut pair, an
inflow strip of 0.5 m^3/s on row 0, and four tires (1.5 m x 2.4 m rectangle,
5 m/s along +z) each with its own 64 x 64 patch of 2 cm cells, dt = 1/120 s.
Synthetic inputs stand in for scenes: the reference publishes no dataset.

Prints one JSON line. `value` is cell-steps/s with the state resident in HBM
(a cell-step = one coarse cell, both layers, one substep; nested 2 cm cells
are counted the same way); `e2e` is the same metric through the public API
with the per-step tire pushes from pinned host memory and the step's spray
events and FP64 ledger read back each step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload grid|batch] [--windows 256] [--batch-tires 1|0]

--workload batch: 256 independent windows, sides log-uniform 64..512 cells of
0.2 m, each with its own seed, 1..4 puddles and 0..4 tires with 64 x 64
patches, all stepped together (silt_batch_step); a step advances every window.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "dirty-gen_b200"))

RES = 2048
CELL = 0.2
DT = 1.0 / 120.0
FINE_RES = 64
INFLOW = (0, -2.0, 2.0, 0.5)
# Algorithmic bytes of k_force per stepped cell-layer: water reads h, u, v,
# bed (16 B) and writes u, v (8 B); slurry also reads grain and moisture (5 B).
FORCE_BYTES_WATER = 24
FORCE_BYTES_SLURRY = 29
STEP_BYTES_PER_CELL = 57   # the fused step's algorithmic bytes (both layers) per coarse cell
# Per stepped cell-layer and substep, as each layer steps on its own: water
# reads h, u, v, bed and writes h, u, v; slurry also reads grain and moisture.
STEP_BYTES_WATER = 28
STEP_BYTES_SLURRY = 33


BATCH_PHASES = ["closure crops + wake entrainment", "per-window planning (workers)", "nested patch launches",
                "coarse pair + open water", "patch peel", "tracers + reach", "closure correction + books"]


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--res", type=int, default=RES)
    ap.add_argument("--no-tires", action="store_true")
    ap.add_argument("--no-baseline", action="store_true")
    ap.add_argument("--no-batch-roofline", action="store_true",
                    help="grid: skip the second roofline entry (the batched force kernel on the 256-window batch)")
    ap.add_argument("--workload", default="grid", choices=["grid", "batch", "window200", "walls200", "closure"],
                    help="grid: one 2048^2 grid with four tire patches; batch: many windows stepped together; "
                         "window200: the reference's own 200^2 window, no tires; walls200: that window with a "
                         "current and a vehicle's belly and four wheel contacts as walls; closure: 200^2 windows with "
                         "four tires each, the learned closure against the nested 2 cm sheets")
    ap.add_argument("--windows", type=int, default=None, help="batch: number of windows (256); closure: (128)")
    ap.add_argument("--batch-tires", type=int, default=1, help="batch: 1 = each window's 0..4 tires, 0 = none")
    ap.add_argument("--closure-threshold", type=float, default=0.1,
                    help="closure: residual estimate above which a window's next step runs the nested sheets")
    return ap.parse_args()


def workload(args):
    return {"workload": f"grid{args.res}_8puddles_inflow_4tires64", "res": args.res, "cell_m": CELL,
            "dt_s": DT, "fine_patches": 0 if args.no_tires else 4, "fine_res": FINE_RES,
            "layout": "per_tire64", "l2": "inputs larger than L2 (state ~%d MB)" % (args.res * args.res * 56 // 2**20)}


def make_scene(args):
    import silt_scenes

    return silt_scenes.grid(res=args.res, cell=CELL)


def tires_for(step, args):
    import silt_scenes

    if args.no_tires:
        return []
    return silt_scenes.tires_at(step * DT, speed=5.0)


def seed(core, scene):
    import silt_scenes

    silt_scenes.seed_core(core, scene)
    core.set_inflow(*INFLOW)


def sample_clocks(stop, out, gpu_index):
    q = ("--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    try:
        p = subprocess.Popen(["nvidia-smi", q, "--format=csv,noheader,nounits", "-lms", "100", "-i", str(gpu_index)],
                             stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
    except OSError:
        return
    try:
        while not stop.is_set():
            line = p.stdout.readline()
            if not line:
                break
            out.append(line.strip())
    finally:
        p.terminate()
        try:
            p.wait(timeout=2)
        except subprocess.TimeoutExpired:
            p.kill()


def summarise_clocks(lines):
    sm, mx, reasons = [], 0.0, set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for ln in lines:
        f = [x.strip() for x in ln.split(",")]
        if len(f) < 9:
            continue
        try:
            sm.append(float(f[1]))
            mx = max(mx, float(f[2]))
        except ValueError:
            continue
        for k, name in enumerate(names):
            if f[5 + k].lower().startswith("active"):
                reasons.add(name)
    return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None, "reasons": sorted(reasons),
            "samples": len(sm)}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def host_cpu():
    """The host CPU the CPU legs ran on: model name and logical cores."""
    model = "unknown"
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                model = ln.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return {"model": model, "nproc": os.cpu_count()}


def cpu_threads(args):
    """Threads the oracle runs on: the coarse pair on two (the reference's
    rayon::join of the two sheets), each fine patch's two sheets on their own."""
    return 2 if args.no_tires else 2 * 4


def cpu_baseline(args, scene, max_steps=40, warmup=1, budget_s=15.0, single=True):
    """The CPU oracle (restated reference) on this host: the same workload for a
    bounded sample of steps (at most `max_steps`, stopping once `budget_s` has
    passed), built -O3 -march=native here. Two variants: the reference's
    threading (the two sheets of each pair on their own threads, as its
    rayon::join does) and, with `single`, one thread."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    flags = oracle.use_native_build()

    def run(threads):
        core = oracle.Core(res=args.res, cell=CELL, fine_res=FINE_RES, fine_cell=0.02, layout=1, threads=threads)
        seed(core, scene)
        k = 0
        for _ in range(max(1, warmup)):
            for t in tires_for(k, args):
                core.push_tire(**t)
            core.step(DT)
            k += 1
        steps = 0
        t0 = time.perf_counter()
        el = 0.0
        while steps < max(1, max_steps) and el < budget_s:
            for t in tires_for(k, args):
                core.push_tire(**t)
            core.step(DT)
            k += 1
            steps += 1
            el = time.perf_counter() - t0
        return steps, el

    fine_cells = 0 if args.no_tires else 4 * FINE_RES * FINE_RES
    cells = args.res * args.res + fine_cells
    threads = cpu_threads(args)
    steps, el = run(threads)
    out = {"value": cells * steps / el, "unit": "cell-steps/s", "cores": threads, "kind": "port",
           "steps": steps, "seconds": el, "host": host_cpu(), "build": flags,
           "sample": f"{steps} steps of the same {args.res}^2 workload after {max(1, warmup)} warm-up step(s); "
                     f"coarse pair on 2 threads, fine patch sheets on {threads} ({el:.2f} s)"}
    if single:
        s1, e1 = run(1)
        out["single_thread"] = {"value": cells * s1 / e1, "unit": "cell-steps/s", "cores": 1, "steps": s1,
                                "seconds": e1, "ms_per_step": 1000.0 * e1 / s1}
    return out


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    scene = make_scene(args)
    base = cpu_baseline(args, scene, max_steps=args.steps, warmup=args.warmup, budget_s=60.0, single=False)
    fine_cells = 0 if args.no_tires else 4 * FINE_RES * FINE_RES
    line = {"metric": "cell-steps/s", "value": base["value"], "unit": "cell-steps/s", "n_gpus": args.gpus,
            "steps": base["steps"], "warmup": max(1, args.warmup),
            "ms_per_step": 1000.0 * (args.res * args.res + fine_cells) / base["value"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "impl": "reference", "config": workload(args), "cpu_baseline": base,
            "e2e": {"value": base["value"], "unit": "cell-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_b200(args):
    import numpy as np
    import torch

    import silt_b200

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    stream = torch.cuda.Stream()
    scene = make_scene(args)
    fine_cells = 0 if args.no_tires else 4 * FINE_RES * FINE_RES
    cells_per_step = args.res * args.res + fine_cells
    sheet = silt_b200.Sheet(res=args.res, cell=CELL, fine_res=FINE_RES, fine_cell=0.02,
                            layout=silt_b200.FINE_PER_TIRE, device=local, stream=stream.cuda_stream)
    seed(sheet, scene)
    step_no = 0

    def step_on(sh, n, want_spray):
        for t in tires_for(n, args):
            sh.push_tire(**t)
        return sh.step(DT, want_spray=want_spray)

    def one_step(want_spray):
        nonlocal step_no
        step_no += 1
        return step_on(sheet, step_no, want_spray)

    for _ in range(max(3, args.warmup)):
        one_step(False)
    sheet.sync()
    torch.cuda.synchronize()
    # Device-resident timed region: K steps, no events inside; the library's
    # counters (launches, stepped tiles) are read before and after it.
    p0 = sheet.step_parts()
    stop = threading.Event()
    clock_lines = []
    th = threading.Thread(target=sample_clocks, args=(stop, clock_lines, local), daemon=True)
    th.start()
    time.sleep(0.3)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    h0 = time.perf_counter()
    for _ in range(args.steps):
        one_step(False)
    host_ms = (time.perf_counter() - h0) * 1000.0 / args.steps
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    stop.set()
    th.join(timeout=5)
    p1 = sheet.step_parts()
    parts = {k: p1[k] - p0[k] for k in ("launches", "force_launches", "force_cells", "force_cells_water",
                                        "device_counts", "steps", "sweep_launches", "sweep_solves",
                                        "sweep_local_passes")}
    parts["sweep_passes_max"] = p1["sweep_passes_max"]
    parts["sweep_fallbacks"] = p1["sweep_fallbacks"]
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * cells_per_step * args.steps / (ms / 1000.0)
    # Kernel pass: the same K steps again with two CUDA events around every
    # launch on its stream, for each kernel's device time and share.
    silt_b200.set_kernel_timing(True)
    for _ in range(args.steps):
        one_step(False)
    kt = silt_b200.kernel_times()
    silt_b200.set_kernel_timing(False)
    # Host pass: the library's own clock around its host work in silt_step
    # (planning, uploads, launch submission), to compare with the device time.
    sheet.set_step_timing(True)  # starts the step parts from zero
    host_steps = min(args.steps, 50)
    for _ in range(host_steps):
        one_step(False)
    torch.cuda.synchronize()
    hp = sheet.step_parts()
    sheet.set_step_timing(False)
    host_inside = {"silt_step": hp["host_step_ms"] / host_steps,
                   "nested_patch_planning": hp["host_fine_ms"] / host_steps, "steps": host_steps,
                   "phases": [round(x / host_steps, 4) for x in hp["host_phase_ms"][:7]],
                   "phase_names": BATCH_PHASES}
    # End to end through the public API, every timed step: the tire pushes go
    # in (inside silt_step, from its pinned step table), the spray events and
    # the FP64 ledger come back, and the ledger's closure is checked each step.
    # A second sheet, seeded and warmed up the same way, takes the timed loop's
    # own steps (the cost of a step changes as the water and silt spread).
    sheet.close()
    sheet = silt_b200.Sheet(res=args.res, cell=CELL, fine_res=FINE_RES, fine_cell=0.02,
                            layout=silt_b200.FINE_PER_TIRE, device=local, stream=stream.cuda_stream)
    seed(sheet, scene)
    for n in range(1, max(3, args.warmup) + 1):
        step_on(sheet, n, False)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    e2e_steps = args.steps
    prev = sheet.ledger()
    f0.record(stream)
    nev = 0
    gaps = []   # per step: |(total + cut - opened) now - before| / total, the FP64 books' closure
    rgaps = []  # the same with the transport rounding book taken off
    for n in range(max(3, args.warmup) + 1, max(3, args.warmup) + 1 + e2e_steps):
        ev = step_on(sheet, n, True)
        nev += len(ev)
        led = sheet.ledger()
        kept = led["total_m3"] + led["cut_m3"] - led["opened_m3"]
        kept0 = prev["total_m3"] + prev["cut_m3"] - prev["opened_m3"]
        gaps.append(abs(kept - kept0) / led["total_m3"])
        rgaps.append(abs((kept - led["round_m3"]) - (kept0 - prev["round_m3"])) / led["total_m3"])
        prev = led
    f1.record(stream)
    torch.cuda.synchronize()
    ems = f0.elapsed_time(f1)
    if dist:
        t = torch.tensor([ems], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ems = float(t.item())
    e2e_value = world * cells_per_step * e2e_steps / (ems / 1000.0)
    led = sheet.ledger()
    if rank == 0:
        peak, peak_kind = measured_peak()
        launches = max(parts["force_launches"], 1)
        cw = parts["force_cells_water"] / launches          # stepped cell-layers per coarse substep
        cs = (parts["force_cells"] - parts["force_cells_water"]) / launches
        substeps_per_step = parts["force_launches"] / max(parts["steps"], 1)
        fine_layers = 0 if args.no_tires else 4 * FINE_RES * FINE_RES  # per layer, one patch pass
        models = kernel_bytes_models(cw, cs, fine_layers)
        roof, kernels = kernel_roofline(kt, models, peak, peak_kind)
        step_bytes = substeps_per_step * (STEP_BYTES_WATER * cw + STEP_BYTES_SLURRY * cs) + \
            (STEP_BYTES_WATER + STEP_BYTES_SLURRY) * fine_layers
        step_ms = ms / args.steps
        roof["step"] = {"algorithmic_bytes_per_step": step_bytes, "ms_per_step": step_ms,
                        "achieved": step_bytes / (step_ms / 1000.0) / 1e9, "unit": "GB/s",
                        "frac": step_bytes / (step_ms / 1000.0) / 1e9 / peak,
                        "basis": "28 B per stepped water cell-layer, 33 B per slurry cell-layer per substep "
                                 "(reads h, u, v, bed [+ grain, moisture], writes h, u, v), coarse tiles the "
                                 "step stepped plus every 2 cm patch cell"}
        stepped_per_step = substeps_per_step * (cw + cs) + 2 * fine_layers
        line = {"metric": "cell-steps/s", "value": value, "unit": "cell-steps/s", "n_gpus": world,
                "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": step_ms,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic", "config": workload(args), "roofline": roof, "kernels": kernels,
                "stepped_cell_layers_per_s": world * stepped_per_step * args.steps / (ms / 1000.0),
                "e2e": {"value": e2e_value, "unit": "cell-steps/s", "h2d_bytes_per_step": len(tires_for(1, args)) * 32,
                        "d2h_bytes_per_step": 56 + 4 + 32 * (nev // max(e2e_steps, 1)), "steps": e2e_steps},
                "gpu_launches": int(parts["launches"]), "clocks": summarise_clocks(clock_lines),
                "host_submit_ms_per_step": host_ms,
                "host_ms_inside_silt_step": host_inside,
                "device_counted_steps": int(parts["device_counts"]),
                "confinement": {"form": "gauss-seidel sweep (step_pair)",
                                "most_fixed_point_passes": int(parts["sweep_passes_max"]),
                                "sequential_fallbacks": int(parts["sweep_fallbacks"]),
                                "tile_solves_per_launch": int(parts["sweep_solves"]) / max(int(parts["sweep_launches"]), 1),
                                "local_passes_per_solve": int(parts["sweep_local_passes"]) / max(int(parts["sweep_solves"]), 1)},
                "window_steps_per_s": world * args.steps / (ms / 1000.0),
                "ledger": {"water_m3": led["water_m3"], "slurry_m3": led["slurry_m3"], "opened_m3": led["opened_m3"],
                           "spray_m3": led["spray_m3"], "cut_m3": led["cut_m3"],
                           "gap_max_per_step": max(gaps), "gap_median_per_step": statistics.median(gaps),
                           "gap_steps": len(gaps), "gap_target": 1e-9, "round_m3": led["round_m3"],
                           "gap_max_per_step_after_rounding_book": max(rgaps),
                           "gap_what": "per step |(total + cut - opened) now - before| / total; the f32 transport "
                                       "updates' own rounding is booked in FP64 (round_m3) and taken off in the "
                                       "second figure"}}
        if not args.no_batch_roofline and world == 1:
            sheet.sync()
            line["roofline_batch"] = batch_roofline(args, local, peak, peak_kind)
        if not args.no_baseline:
            line["cpu_baseline"] = cpu_baseline(args, scene)
        print(json.dumps(line), flush=True)
    sheet.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def kernel_bytes_models(cw, cs, fine_layers):
    """Algorithmic bytes of one launch, by kernel name, for the grid step:
    cw, cs = stepped water and slurry cell-layers of one coarse substep,
    fine_layers = 2 cm patch cells per layer."""
    force = FORCE_BYTES_WATER * cw + FORCE_BYTES_SLURRY * cs
    window = (STEP_BYTES_WATER + STEP_BYTES_SLURRY) * fine_layers
    return {"k_force_sweep": (force, "24 B per stepped water cell-layer, 29 B per slurry cell-layer: reads h, u, v, "
                                     "bed (+ grain, moisture), writes u, v"),
            "k_force": (force, "as k_force_sweep"),
            "k_transport": (16 * (cw + cs), "16 B per stepped cell-layer: reads h, u, v, writes h"),
            "k_window_step": (window, "28 B per 2 cm water cell, 33 B per slurry cell (reads h, u, v, bed [+ grain, "
                                      "moisture], writes h, u, v), every patch cell of both layers")}


def kernel_roofline(kt, models, peak, peak_kind):
    """The roofline of the kernel with the largest device time in the kernel
    pass, and every kernel's launches, average and share."""
    total = sum(k["ms"] for k in kt) or 1.0
    kernels = [{"name": k["name"], "launches": k["launches"], "avg_ms": k["ms"] / max(k["launches"], 1),
                "share": k["ms"] / total} for k in kt]
    roof = {"bound": "hbm", "peak": peak, "unit": "GB/s", "peak_kind": peak_kind,
            "timing": "CUDA events around every launch on its stream, in a pass of the same K steps after the "
                      "timed one"}
    if kt:
        top = kt[0]
        short = top["name"].split("::")[-1]
        roof["kernel"] = top["name"]
        roof["share"] = top["ms"] / total
        avg_ms = top["ms"] / max(top["launches"], 1)
        roof["avg_launch_ms"] = avg_ms
        model = models.get(short)
        if model:
            roof["algorithmic_bytes_per_launch"] = model[0]
            roof["bytes_basis"] = model[1]
            roof["achieved"] = model[0] / (avg_ms / 1000.0) / 1e9
            roof["frac"] = roof["achieved"] / peak
        else:
            roof["achieved"] = roof["frac"] = None
        roof["traffic"] = profiled_kernel_traffic(short)
    return roof, kernels


def profiled_kernel_traffic(short):
    """DRAM bytes per launch (read + write) of the kernel from the committed
    ncu summary profiles/kernel_traffic.txt (lines `name: bytes`), or None."""
    try:
        for ln in open(os.path.join(ROOT, "profiles", "kernel_traffic.txt")):
            if ln.split(":", 1)[0].strip() == short:
                return float(ln.split(":", 1)[1].split()[0])
    except (OSError, ValueError, IndexError):
        pass
    return None


def batch_roofline(args, local, peak, peak_kind):
    """The batched force kernel on the 256-window batch (sides log-uniform
    64..512, 0..4 tires): its kernel pass and roofline."""
    import numpy as np
    import torch

    import silt_b200
    import silt_scenes

    stream = torch.cuda.Stream()
    wins = silt_scenes.batch_windows(n=256, base_seed=0x9E3779B9, cell=CELL)
    sheets = []
    for w in wins:
        sh = silt_b200.Sheet(res=w["res"], cell=CELL, fine_res=FINE_RES, fine_cell=0.02,
                             layout=silt_b200.FINE_PER_TIRE, device=local, stream=stream.cuda_stream,
                             engine=silt_b200.ENGINE_GRID)
        silt_scenes.seed_core(sh, w)
        sheets.append(sh)
    batch = silt_b200.Batch(sheets)
    step_no = 0

    def one_step():
        nonlocal step_no
        step_no += 1
        idx, ts = [], []
        for k, w in enumerate(wins):
            for t in batch_tires(step_no, w):
                idx.append(k)
                ts.append(t)
        batch.push_tires(idx, ts)
        batch.step(DT)

    for _ in range(3):
        one_step()
    steps = 10
    p0 = batch.parts()
    silt_b200.set_kernel_timing(True)
    for _ in range(steps):
        one_step()
    kt = silt_b200.kernel_times()
    silt_b200.set_kernel_timing(False)
    p1 = batch.parts()
    launches = max(p1["force_launches"] - p0["force_launches"], 1)
    cw = (p1["force_cells_water"] - p0["force_cells_water"]) / launches
    cs = (p1["force_cells"] - p1["force_cells_water"] - (p0["force_cells"] - p0["force_cells_water"])) / launches
    force = FORCE_BYTES_WATER * cw + FORCE_BYTES_SLURRY * cs
    out = {"workload": "batch256_side64-512_logu_1-4puddles_0-4tires64", "steps": steps}
    for k in kt:
        short = k["name"].split("::")[-1]
        if short in ("k_batch_force_sweep", "k_batch_force"):
            avg = k["ms"] / max(k["launches"], 1)
            out.update({"kernel": k["name"], "avg_launch_ms": avg, "algorithmic_bytes_per_launch": force,
                        "stepped_cell_layers_per_launch": cw + cs, "achieved": force / (avg / 1000.0) / 1e9,
                        "peak": peak, "unit": "GB/s", "peak_kind": peak_kind,
                        "share": k["ms"] / (sum(x["ms"] for x in kt) or 1.0),
                        "traffic": profiled_kernel_traffic(short)})
            out["frac"] = out["achieved"] / peak
    out["kernels"] = [{"name": k["name"], "launches": k["launches"], "avg_ms": k["ms"] / max(k["launches"], 1)}
                      for k in kt[:8]]
    batch.close()
    for sh in sheets:
        sh.close()
    return out


# ---------------------------------------------------------------- batched windows

def batch_workload(args):
    return {"workload": f"batch{args.windows}_side64-512_logu_1-4puddles_" +
                        ("0-4tires64" if args.batch_tires else "notires"),
            "windows": args.windows, "cell_m": CELL, "dt_s": DT, "fine_res": FINE_RES, "layout": "per_tire64",
            "l2": "inputs larger than L2 (state ~1 GB)"}


def batch_scene(args, rank=0):
    import silt_scenes

    wins = silt_scenes.batch_windows(n=args.windows, base_seed=0x9E3779B9 + 1000003 * rank, cell=CELL)
    if not args.batch_tires:
        for w in wins:
            w["tires"] = 0
    return wins


def batch_tires(step, win):
    import silt_scenes

    if not win["tires"]:
        return []
    return silt_scenes.tires_at(step * DT, speed=5.0, z0=-0.5 * win["res"] * CELL)[:win["tires"]]


def batch_cells(wins):
    return sum(w["res"] * w["res"] + w["tires"] * FINE_RES * FINE_RES for w in wins)


def batch_cpu(args, wins, max_steps, warmup, budget_s):
    """The oracle on a bounded sample of the batch: every 16th window, each
    stepped on its own (the reference steps one FluidCore at a time)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    oracle.use_native_build()
    import silt_scenes

    sample = wins[::16]
    cores = []
    for w in sample:
        c = oracle.Core(res=w["res"], cell=CELL, fine_res=FINE_RES, fine_cell=0.02, layout=1, threads=2)
        silt_scenes.seed_core(c, w)
        cores.append(c)
    k = 0
    for _ in range(max(1, warmup)):
        k += 1
        for w, c in zip(sample, cores):
            for t in batch_tires(k, w):
                c.push_tire(**t)
            c.step(DT)
    steps = 0
    t0 = time.perf_counter()
    el = 0.0
    while steps < max(1, max_steps) and el < budget_s:
        k += 1
        for w, c in zip(sample, cores):
            for t in batch_tires(k, w):
                c.push_tire(**t)
            c.step(DT)
        steps += 1
        el = time.perf_counter() - t0
    value = batch_cells(sample) * steps / el
    return {"value": value, "unit": "cell-steps/s", "cores": 2, "kind": "port", "steps": steps, "seconds": el, "host": host_cpu(),
            "sample": f"{len(sample)} of the {len(wins)} windows (every 16th), {steps} steps after "
                      f"{max(1, warmup)} warm-up step(s), one window at a time, each pair on 2 threads ({el:.2f} s)"}


def run_batch_reference(args):
    if int(os.environ.get("RANK", "0")) != 0:
        return
    wins = batch_scene(args)
    base = batch_cpu(args, wins, max_steps=args.steps, warmup=args.warmup, budget_s=60.0)
    line = {"metric": "cell-steps/s", "value": base["value"], "unit": "cell-steps/s", "n_gpus": args.gpus,
            "steps": base["steps"], "warmup": max(1, args.warmup),
            "ms_per_step": 1000.0 * batch_cells(wins) / base["value"], "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": batch_workload(args), "cpu_baseline": base,
            "e2e": {"value": base["value"], "unit": "cell-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_batch(args):
    import torch

    import silt_b200
    import silt_scenes

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    stream = torch.cuda.Stream()
    import silt_shard

    all_wins = batch_scene(args)
    mine = silt_shard.shard(len(all_wins), rank, world)  # round-robin: windows are independent
    wins = [all_wins[w] for w in mine]
    sheets = []
    for w in wins:
        sh = silt_b200.Sheet(res=w["res"], cell=CELL, fine_res=FINE_RES, fine_cell=0.02,
                             layout=silt_b200.FINE_PER_TIRE, device=local, stream=stream.cuda_stream,
                             engine=silt_b200.ENGINE_GRID)
        silt_scenes.seed_core(sh, w)
        sheets.append(sh)
    batch = silt_b200.Batch(sheets)
    cells = batch_cells(wins)
    step_no = 0
    # Every window's tires as one record array: the same pushes batch_tires
    # gives, with z advanced in place each step (float32, as tires_at does).
    import numpy as np

    f32 = np.float32
    idx, recs, zbase, zrow = [], [], [], []
    for k, w in enumerate(wins):
        for q, t in enumerate(batch_tires(0, w)):
            idx.append(k)
            recs.append(t)
            zbase.append(f32(0.0) + f32(-0.5 * w["res"] * CELL))  # center z + z0, as tires_at sums them
            zrow.append(f32((-0.5, -0.5, 0.5, 0.5)[q] * 2.4))       # the tire's offset along the wheelbase
    idx = np.asarray(idx, np.int32)
    push_rec = np.zeros(len(recs), silt_b200.TIRE_DTYPE)
    for name in silt_b200.TIRE_DTYPE.names:
        push_rec[name] = [r[name] for r in recs]
    zbase = np.asarray(zbase, f32)
    zrow = np.asarray(zrow, f32)

    def one_step():
        nonlocal step_no
        step_no += 1
        push_rec["z"] = (zbase + f32(5.0) * f32(step_no * DT)) + zrow
        batch.push_tires(idx, push_rec)
        batch.step(DT)

    # The launch settings come from the library's autotuner, which times the
    # first steps under each candidate (every candidate gives the same bits);
    # the warm-up steps follow once it has chosen.
    batch.autotune(True)
    for _ in range(40):
        if batch.tune()["tuned"]:
            break
        one_step()
    for _ in range(max(3, args.warmup)):
        one_step()
    torch.cuda.synchronize()
    stop = threading.Event()
    clock_lines = []
    th = threading.Thread(target=sample_clocks, args=(stop, clock_lines, local), daemon=True)
    th.start()
    time.sleep(0.3)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    h0 = time.perf_counter()
    for _ in range(args.steps):
        one_step()
    host_ms = (time.perf_counter() - h0) * 1000.0 / args.steps
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    # The library's step parts (events around the force and transport
    # launches, host clocks per phase) in a pass of their own after the timed
    # one, whose region they would otherwise slow; per-step figures below.
    batch.set_timing(True)
    part_steps = min(args.steps, 10)
    for _ in range(part_steps):
        one_step()
    torch.cuda.synchronize()
    parts = batch.parts()
    batch.set_timing(False)
    parts = {k: ([x * args.steps / part_steps for x in v] if isinstance(v, list) else v * args.steps / part_steps)
             for k, v in parts.items()}
    # Kernel pass: CUDA events around every launch, each kernel's device time.
    silt_b200.set_kernel_timing(True)
    for _ in range(part_steps):
        one_step()
    kt = silt_b200.kernel_times()
    silt_b200.set_kernel_timing(False)
    ktotal = sum(k["ms"] for k in kt) or 1.0
    kernels = [{"name": k["name"], "launches": k["launches"], "avg_ms": k["ms"] / max(k["launches"], 1),
                "ms_per_step": k["ms"] / part_steps, "share": k["ms"] / ktotal} for k in kt[:16]]
    stop.set()
    th.join(timeout=5)
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    total_cells = batch_cells(all_wins)
    value = total_cells * args.steps / (ms / 1000.0)
    # End to end: the pushes in, every window's FP64 ledger back (gathered
    # over the ranks: the one collective), each step.
    e2e_steps = max(5, args.steps // 4)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(e2e_steps):
        one_step()
        table = silt_shard.gather_ledger_rows(mine, batch.ledger_rows(), len(all_wins), dist,
                                              device="cuda" if dist else "cpu")
    f1.record(stream)
    torch.cuda.synchronize()
    ems = f0.elapsed_time(f1)
    if dist:
        t = torch.tensor([ems], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ems = float(t.item())
    e2e_value = total_cells * e2e_steps / (ems / 1000.0)
    if rank == 0:
        peak, peak_kind = measured_peak()
        launches = max(parts["force_launches"], 1)
        force_ms = parts["force_ms"] / launches
        cw = parts["force_cells_water"] / launches
        cs = (parts["force_cells"] - parts["force_cells_water"]) / launches
        force_bytes = FORCE_BYTES_WATER * cw + FORCE_BYTES_SLURRY * cs
        achieved = force_bytes / (force_ms / 1000.0) / 1e9 if force_ms > 0 else None
        coarse = sum(w["res"] * w["res"] for w in wins)
        roof = {"bound": "hbm", "kernel": "k_batch_force", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak if achieved else None, "peak_kind": peak_kind, "traffic": None,
                "algorithmic_bytes_per_launch": force_bytes, "avg_launch_ms": force_ms,
                "stepped_cell_layers_per_launch": cw + cs, "active_fraction": (cw + cs) / (2.0 * coarse),
                "transport_avg_launch_ms": parts["transport_ms"] / launches}
        n_tires = sum(w["tires"] for w in wins)
        line = {"metric": "cell-steps/s", "value": value, "unit": "cell-steps/s", "n_gpus": world,
                "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": ms / args.steps,
                "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic", "config": batch_workload(args), "roofline": roof,
                "e2e": {"value": e2e_value, "unit": "cell-steps/s", "h2d_bytes_per_step": 32 * n_tires,
                        "d2h_bytes_per_step": 40 * len(wins), "steps": e2e_steps},
                "gpu_launches": int(parts["launches"]), "kernels": kernels, "launch_settings": batch.tune(),
                "confinement": {"form": "gauss-seidel sweep (step_pair)",
                                "most_fixed_point_passes": int(parts["sweep_passes_max"] * part_steps / args.steps),
                                "tile_solves_per_launch": parts["sweep_solves"] / max(parts["sweep_launches"], 1),
                                "local_passes_per_solve": parts["sweep_local_passes"] / max(parts["sweep_solves"], 1)},
                "clocks": summarise_clocks(clock_lines),
                "host_submit_ms_per_step": host_ms,
                "host_ms_per_step": {"batch_step": parts["host_step_ms"] / args.steps,
                                     "per_window_before_coarse": parts["host_fine_ms"] / args.steps,
                                     "phases": [round(x / args.steps, 4) for x in parts["host_phase_ms"][:7]],
                                     "phase_names": BATCH_PHASES},
                "window_steps_per_s": len(all_wins) * args.steps / (ms / 1000.0),
                "windows": len(all_wins), "windows_rank0": len(wins), "coarse_cells_rank0": coarse,
                "tires_rank0": n_tires, "ledger_total_m3": float(table[:, 6].sum())}
        if not args.no_baseline:
            line["cpu_baseline"] = batch_cpu(args, all_wins, max_steps=20, warmup=1, budget_s=20.0)
        print(json.dumps(line), flush=True)
    batch.close()
    for sh in sheets:
        sh.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


# ---------------------------------------------------------------- the 200 x 200 window

def run_window200(args):
    """The reference's CPU-runnable case: one 200 x 200 window (0.2 m cells),
    ruts, a Gaussian puddle and a rut slurry film, no tires, dt = 1/120 s,
    stepped on the window engine (the exact box-by-box step). walls200 adds a
    uniform current and a standing vehicle's belly and wheel contacts as
    walls (the walled step, mask and displacement every step, scour)."""
    import torch

    import silt_b200
    import silt_scenes

    if int(os.environ.get("RANK", "0")) != 0 and args.impl == "reference":
        return
    scene = silt_scenes.window200()
    res = scene["res"]
    walled = args.workload == "walls200"
    seed_window = silt_scenes.seed_walled if walled else silt_scenes.seed_core
    cfgw = {"workload": "window200_ruts_puddle_slurry" + ("_current_belly_4wheels" if walled else ""), "res": res,
            "cell_m": CELL, "dt_s": DT, "engine": "window", "l2": "state fits in L2 (~2 MB); no flush between steps"}
    if args.impl == "reference":
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        oracle.use_native_build()

        core = oracle.Core(threads=2)
        seed_window(core, scene)
        for _ in range(max(1, args.warmup)):
            core.step(DT)
        steps, t0, el = 0, time.perf_counter(), 0.0
        while steps < max(1, args.steps) and el < 60.0:
            core.step(DT)
            steps += 1
            el = time.perf_counter() - t0
        v = res * res * steps / el
        base = {"value": v, "unit": "cell-steps/s", "cores": 2, "kind": "port", "steps": steps, "seconds": el,
                "host": host_cpu(),
                "sample": f"{steps} steps after {max(1, args.warmup)} warm-up, the pair on 2 threads ({el:.2f} s)"}
        print(json.dumps({"metric": "cell-steps/s", "value": v, "unit": "cell-steps/s", "n_gpus": args.gpus,
                          "steps": steps, "warmup": max(1, args.warmup), "ms_per_step": 1000.0 * el / steps,
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                          "data": "synthetic", "impl": "reference", "config": cfgw, "cpu_baseline": base,
                          "window_steps_per_s": steps / el,
                          "e2e": {"value": v, "unit": "cell-steps/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}), flush=True)
        return
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    stream = torch.cuda.Stream()
    sheet = silt_b200.Sheet(device=local, stream=stream.cuda_stream)
    seed_window(sheet, scene)
    for _ in range(max(3, args.warmup)):
        sheet.step(DT, want_spray=False)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        sheet.step(DT, want_spray=False)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    # The library's step parts in a pass of their own (timing mode reads back
    # each step's Gauss-Seidel pass count, which waits for the step).
    sheet.set_step_timing(True)
    part_steps = min(args.steps, 20)
    for _ in range(part_steps):
        sheet.step(DT, want_spray=False)
    torch.cuda.synchronize()
    parts = sheet.step_parts()
    sheet.set_step_timing(False)
    gs = {"most_passes": int(parts["sweep_passes_max"]),
          "mean_passes_per_layer_step": parts["sweep_local_passes"] / max(parts["sweep_solves"], 1),
          "sequential_fallbacks": int(parts["sweep_fallbacks"]), "steps": part_steps}
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    e2e_steps = max(10, args.steps // 4)
    f0.record(stream)
    for _ in range(e2e_steps):
        sheet.step(DT)
        sheet.ledger()
    f1.record(stream)
    torch.cuda.synchronize()
    ems = f0.elapsed_time(f1)
    line = {"metric": "cell-steps/s", "value": res * res * args.steps / (ms / 1000.0), "unit": "cell-steps/s",
            "n_gpus": 1, "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": cfgw, "window_steps_per_s": args.steps / (ms / 1000.0),
            "e2e": {"value": res * res * e2e_steps / (ems / 1000.0), "unit": "cell-steps/s",
                    "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 60, "steps": e2e_steps},
            "gpu_launches": int(parts["launches"]) * args.steps // max(part_steps, 1),
            "gauss_seidel": gs}
    if not args.no_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        oracle.use_native_build()

        core = oracle.Core(threads=2)
        seed_window(core, scene)
        core.step(DT)
        t0 = time.perf_counter()
        for _ in range(20):
            core.step(DT)
        el = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": res * res * 20 / el, "unit": "cell-steps/s", "cores": 2, "kind": "port",
                                "host": host_cpu(),
                                "sample": f"20 steps after 1 warm-up, the pair on 2 threads ({el:.2f} s)"}
    print(json.dumps(line), flush=True)
    sheet.close()


CLOSURE_EVAL_SEED = 0xC0FFEE11  # evaluation windows: not among the training windows


def closure_workload(args):
    return {"workload": f"closure{args.windows}_win200_4tires_speed2-10", "windows": args.windows, "res": 200,
            "cell_m": CELL, "dt_s": DT, "fine_res": FINE_RES, "layout": "per_tire64",
            "network": "3x3 conv 6(16)-32-32-4(16), bf16, fp32 accumulate", "crop": 32,
            "residual_threshold": args.closure_threshold,
            "l2": "inputs larger than L2 (four forms x 128 windows, ~0.7 GB of state)"}


def closure_push_records(scenes, silt_b200, T):
    """Every window's four tires as one record array, with what tires_at adds
    to z each step kept apart so the per-step z is the same f32 arithmetic."""
    import numpy as np

    f32 = np.float32
    idx, recs, zb, spd, zrow = [], [], [], [], []
    for k, sc in enumerate(scenes):
        for q, t in enumerate(T.scene_tires(sc, 0)):
            idx.append(k)
            recs.append(t)
            zb.append(f32(0.0) + f32(sc["z0"]))
            spd.append(f32(sc["speed"]))
            zrow.append(f32((-0.5, -0.5, 0.5, 0.5)[q] * 2.4))
    rec = np.zeros(len(recs), silt_b200.TIRE_DTYPE)
    for name in silt_b200.TIRE_DTYPE.names:
        rec[name] = [r[name] for r in recs]
    return np.asarray(idx, np.int32), rec, np.asarray(zb, f32), np.asarray(spd, f32), np.asarray(zrow, f32)


def closure_cpu(scenes, T, max_steps, budget_s):
    """The reference's form (nested 2 cm sheets, one window at a time) on the
    oracle for every 16th window."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    oracle.use_native_build()
    import silt_scenes

    sample = scenes[::16]
    cores = []
    for sc in sample:
        c = oracle.Core(res=200, cell=CELL, fine_res=FINE_RES, fine_cell=0.02, layout=1, threads=2)
        silt_scenes.seed_core(c, sc)
        cores.append(c)
    for sc, c in zip(sample, cores):
        for t in T.scene_tires(sc, 1):
            c.push_tire(**t)
        c.step(DT)
    steps, t0, el = 0, time.perf_counter(), 0.0
    while steps < max(1, max_steps) and el < budget_s:
        for sc, c in zip(sample, cores):
            for t in T.scene_tires(sc, 2 + steps):
                c.push_tire(**t)
            c.step(DT)
        steps += 1
        el = time.perf_counter() - t0
    v = len(sample) * steps / el
    return {"value": v, "unit": "window-steps/s", "cores": 2, "kind": "port", "steps": steps, "seconds": el,
            "host": host_cpu(),
            "sample": f"{len(sample)} of the {len(scenes)} windows (every 16th), nested per-tire 64^2 sheets, "
                      f"{steps} steps after 1 warm-up, one window at a time, each pair on 2 threads ({el:.2f} s)"}


def closure_fp64_judge(scenes, T, C, net, zero, forms, steps, every=16, probe_every=5):
    """The closure judged against the FP64 nested-sheet oracle (oracle.Core64:
    the same restated step in double, per-tire 64 x 64 2 cm sheets) on every
    `every`-th window:

    * depth error: relative L2 of both layers' depth after `steps` steps, of
      the closure run and of the f32 GPU nested run, against the FP64 run;
    * flux error: every `probe_every` steps the FP64 state is loaded into two
      GPU windows, one stepped with the closure and one with a zero network
      (the closure's coarse step alone); the correction the closure's face
      transfers make (closure minus uncorrected depth change) is compared with
      the correction the FP64 nested sheets make (FP64 nested minus uncorrected
      depth change) over the window, as a relative L2."""
    import numpy as np
    import torch

    import silt_b200
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    import silt_scenes

    picked = list(range(0, len(scenes), every))
    names = ("water", "slurry", "uw", "vw", "us", "vs")
    num = {"closure": 0.0, "nested_f32": 0.0}
    den = 0.0
    fnum = fden = 0.0
    probes = 0
    for w in picked:
        sc = scenes[w]
        ref = oracle.Core64(res=200, cell=CELL, fine_res=FINE_RES, fine_cell=0.02, layout=1, threads=2)
        silt_scenes.seed_core(ref, sc)
        pair = []
        for nn in (net, zero):
            sh = silt_b200.Sheet(res=200, cell=CELL, fine_res=FINE_RES, fine_cell=0.02,
                                 layout=silt_b200.FINE_PER_TIRE, engine=silt_b200.ENGINE_GRID)
            silt_scenes.seed_core(sh, sc)
            C.set_coupling(sh, C.COUPLING_CLOSURE, nn, 1e30)
            pair.append(sh)
        for k in range(1, steps + 1):
            tires = T.scene_tires(sc, k)
            if (k - 1) % probe_every == 0:
                before = {n: ref.get(n) for n in names}
                for sh in pair:
                    for n in names:
                        sh.set(n, before[n].astype(np.float32))
                    for t in tires:
                        sh.push_tire(**t)
                    sh.step(DT, want_spray=False)
            for t in tires:
                ref.push_tire(**t)
            ref.step(DT)
            if (k - 1) % probe_every == 0:
                for layer in ("water", "slurry"):
                    h0 = before[layer]
                    d_ref = ref.get(layer) - h0
                    d_cl = pair[0].get(layer).astype(np.float64) - h0
                    d_un = pair[1].get(layer).astype(np.float64) - h0
                    target, pred = d_ref - d_un, d_cl - d_un
                    fnum += float(((pred - target) ** 2).sum())
                    fden += float((target ** 2).sum())
                probes += 1
        for layer in ("water", "slurry"):
            y = ref.get(layer)
            den += float((y ** 2).sum())
            for name, key in (("closure", "closure"), ("nested", "nested_f32")):
                x = forms[name][0][w].get(layer).astype(np.float64)
                num[key] += float(((x - y) ** 2).sum())
        for sh in pair:
            sh.close()
    torch.cuda.synchronize()
    return {"oracle": "FP64 restatement of the step (oracle.Core64), nested per-tire 64^2 2 cm sheets",
            "windows": len(picked), "steps": steps,
            "depth_rel_l2_closure": math.sqrt(num["closure"] / den),
            "depth_rel_l2_nested_f32": math.sqrt(num["nested_f32"] / den),
            "flux_correction_rel_l2": math.sqrt(fnum / fden) if fden > 0 else None,
            "flux_probes": probes,
            "flux_what": "closure's depth correction (its face transfers) against the FP64 nested sheets' "
                         "correction of the same coarse step, one step from the FP64 state"}


def run_closure_reference(args):
    if int(os.environ.get("RANK", "0")) != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "dirty-gen_b200"))
    import silt_closure_train as T

    scenes = [T.drive_scene(k, CLOSURE_EVAL_SEED) for k in range(args.windows)]
    base = closure_cpu(scenes, T, args.steps, 60.0)
    line = {"metric": "window-steps/s", "value": base["value"], "unit": "window-steps/s", "n_gpus": args.gpus,
            "steps": base["steps"], "warmup": 1, "ms_per_step": 1000.0 * len(scenes) / base["value"],
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "impl": "reference", "config": closure_workload(args), "cpu_baseline": base,
            "e2e": {"value": base["value"], "unit": "window-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_closure(args):
    """Configuration 5: windows of 200^2 with four tires each (speed U(2, 10)
    m/s), the learned closure against the full nested 64^2 2 cm sheets, from
    the same start with the same tires; window-steps/s of both forms and the
    relative L2 depth error of the closure (and of the plain coarse step)
    against the nested run."""
    import numpy as np
    import torch

    import silt_b200
    import silt_closure as C
    import silt_closure_train as T

    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    wpath = os.path.join(ROOT, "dirty-gen_b200", "closure_weights.npz")
    if not os.path.exists(wpath):
        raise SystemExit(f"{wpath} is missing: train it with dirty-gen_b200/silt_closure_train.py")
    w = np.load(wpath)
    net = C.Closure(w["params"], w["norm"])
    zero = C.Closure(np.zeros(C.NPARAM, np.float32), w["norm"])  # the closure's coarse step with no correction
    scenes = [T.drive_scene(k, CLOSURE_EVAL_SEED) for k in range(args.windows)]
    forms = {}
    for name, mode, nn, thr in (("nested", C.COUPLING_NESTED, None, 0.0),
                                ("closure", C.COUPLING_CLOSURE, net, args.closure_threshold),
                                ("uncorrected", C.COUPLING_CLOSURE, zero, 1e30),
                                ("plain", C.COUPLING_NONE, None, 0.0)):
        sheets = T.make_sheets(scenes, stream.cuda_stream, mode, nn, thr)
        forms[name] = (sheets, silt_b200.Batch(sheets))
    idx, rec, zb, spd, zrow = closure_push_records(scenes, silt_b200, T)
    f32 = np.float32
    step_of = {name: 0 for name in forms}

    def one_step(name):
        step_of[name] += 1
        rec["z"] = (zb + spd * f32(step_of[name] * DT)) + zrow
        b = forms[name][1]
        b.push_tires(idx, rec)
        b.step(DT)

    warm = max(3, args.warmup)
    timed = {}
    parts = {}
    stop = threading.Event()
    clock_lines = []
    th = threading.Thread(target=sample_clocks, args=(stop, clock_lines, 0), daemon=True)
    th.start()
    time.sleep(0.3)
    part_steps = {}
    for name in forms:
        for _ in range(warm):
            one_step(name)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            one_step(name)
        e1.record(stream)
        torch.cuda.synchronize()
        timed[name] = e0.elapsed_time(e1)
        # The library's step parts (per-launch events, host clocks) in a
        # short pass of their own: their events would slow the timed one.
        forms[name][1].set_timing(True)
        part_steps[name] = min(args.steps, 10)
        for _ in range(part_steps[name]):
            one_step(name)
        torch.cuda.synchronize()
        parts[name] = forms[name][1].parts()
        forms[name][1].set_timing(False)
    stop.set()
    th.join(timeout=5)
    # Depth error against the nested run, every window and both layers.
    def rel_l2(a, b):
        num = den = 0.0
        for sa, sb in zip(forms[a][0], forms[b][0]):
            for layer in ("water", "slurry"):
                x, y = sa.plane_device(layer).double(), sb.plane_device(layer).double()
                num += float(((x - y) ** 2).sum())
                den += float((y ** 2).sum())
        return math.sqrt(num / den)

    torch.cuda.synchronize()
    err_closure = rel_l2("closure", "nested")
    err_plain = rel_l2("plain", "nested")
    err_uncorrected = rel_l2("uncorrected", "nested")
    # End to end through the public API: pushes in from host memory and every
    # window's FP64 ledger back each step; the ledger gap per step is checked
    # on the way (volume now against volume before plus what was opened).
    e2e = {}
    gaps = {}
    e2e_steps = max(5, args.steps // 4)
    for name in ("closure", "nested"):
        b = forms[name][1]
        prev = b.ledger_rows()
        worst = 0.0
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for _ in range(e2e_steps):
            one_step(name)
            rows = b.ledger_rows()
            # Books with the dry cut's volume: total + cut - opened is conserved.
            tot, opened = rows[:, 6] + rows[:, 7], rows[:, 5]
            expect = prev[:, 6] + prev[:, 7] + (opened - prev[:, 5])
            worst = max(worst, float(np.max(np.abs(tot - expect) / np.maximum(expect, 1e-30))))
            prev = rows
        f1.record(stream)
        torch.cuda.synchronize()
        e2e[name] = args.windows * e2e_steps / (f0.elapsed_time(f1) / 1000.0)
        gaps[name] = worst
    cs = [C.stats(sh) for sh in forms["closure"][0]]
    n_closure = sum(s["closure_steps"] for s in cs)
    n_fallback = sum(s["fallback_steps"] for s in cs)
    # The network alone on the windows' crops (tensor-core share of the step).
    x = torch.zeros((args.windows, C.CROP, C.CROP, C.CIN), dtype=torch.bfloat16, device="cuda")
    tnet = C.Net(w["params"])
    with torch.cuda.stream(stream):
        for _ in range(3):
            tnet.forward(x)
        g0 = torch.cuda.Event(enable_timing=True)
        g1 = torch.cuda.Event(enable_timing=True)
        reps = 20
        g0.record(stream)
        for _ in range(reps):
            tnet.forward(x)
        g1.record(stream)
    torch.cuda.synchronize()
    cnn_ms = g0.elapsed_time(g1) / reps
    cnn_flops = 2.0 * args.windows * C.CROP * C.CROP * 9 * (C.CIN * C.HID + C.HID * C.HID + C.HID * C.COUT)
    peak, peak_kind = measured_peak()
    bf16_peak = None
    try:
        mp = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        bf16_peak = mp.get("bf16_tflops")
    except Exception:
        pass
    pc = parts["closure"]
    launches = max(pc["force_launches"], 1)
    force_ms = pc["force_ms"] / launches
    cw = pc["force_cells_water"] / launches
    csl = (pc["force_cells"] - pc["force_cells_water"]) / launches
    force_bytes = FORCE_BYTES_WATER * cw + FORCE_BYTES_SLURRY * csl
    achieved = force_bytes / (force_ms / 1000.0) / 1e9 if force_ms > 0 else None
    ws_closure = args.windows * args.steps / (timed["closure"] / 1000.0)
    ws_nested = args.windows * args.steps / (timed["nested"] / 1000.0)
    ws_plain = args.windows * args.steps / (timed["plain"] / 1000.0)
    line = {"metric": "window-steps/s", "value": ws_closure, "unit": "window-steps/s", "n_gpus": 1,
            "steps": args.steps, "warmup": warm, "ms_per_step": timed["closure"] / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32 (network bf16)",
            "data": "synthetic", "config": closure_workload(args),
            "roofline": {"bound": "hbm", "kernel": "k_batch_force", "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak if achieved else None, "peak_kind": peak_kind,
                         "traffic": None, "algorithmic_bytes_per_launch": force_bytes, "avg_launch_ms": force_ms},
            "closure_cnn": {"bound": "tensor", "kernel": "k_conv3x3 (tcgen05)", "flops_per_step": cnn_flops,
                            "ms_per_step": cnn_ms, "achieved_tflops": cnn_flops / (cnn_ms / 1000.0) / 1e12,
                            "peak_tflops": bf16_peak,
                            "frac": (cnn_flops / (cnn_ms / 1000.0) / 1e12) / bf16_peak if bf16_peak else None},
            "e2e": {"value": e2e["closure"], "unit": "window-steps/s", "h2d_bytes_per_step": 32 * len(rec),
                    "d2h_bytes_per_step": 40 * args.windows, "steps": e2e_steps},
            "nested": {"window_steps_per_s": ws_nested, "ms_per_step": timed["nested"] / args.steps,
                       "e2e_window_steps_per_s": e2e["nested"], "ledger_gap_max": gaps["nested"]},
            "plain_coarse": {"window_steps_per_s": ws_plain, "ms_per_step": timed["plain"] / args.steps,
                             "depth_rel_l2_vs_nested": err_plain,
                             "what": "no sheets, tires shove the 20 cm cells"},
            "uncorrected": {"window_steps_per_s": args.windows * args.steps / (timed["uncorrected"] / 1000.0),
                            "depth_rel_l2_vs_nested": err_uncorrected,
                            "what": "the closure's coarse step with a zero network (no tire effect)"},
            "speedup_vs_nested": ws_closure / ws_nested,
            "depth_rel_l2_vs_nested": err_closure,
            "ledger_gap_max": gaps["closure"],
            "closure_steps": n_closure, "fallback_steps": n_fallback,
            "steps_compared": warm + args.steps + part_steps["closure"],
            "gpu_launches": int(pc["launches"]) * args.steps // max(part_steps["closure"], 1),
            "host_ms_per_step": {name: {"step": parts[name]["host_step_ms"] / max(part_steps[name], 1),
                                        "phases": [round(x / max(part_steps[name], 1), 4)
                                                   for x in parts[name]["host_phase_ms"][:7]]}
                                 for name in forms},
            "host_phase_names": BATCH_PHASES,
            "clocks": summarise_clocks(clock_lines)}
    assert step_of["closure"] == step_of["nested"]
    line["vs_fp64_nested"] = closure_fp64_judge(scenes, T, C, net, zero, forms, step_of["closure"])
    if not args.no_baseline:
        line["cpu_baseline"] = closure_cpu(scenes, T, 40, 20.0)
    print(json.dumps(line), flush=True)
    for name in forms:
        forms[name][1].close()
        for sh in forms[name][0]:
            sh.close()
    net.close()
    zero.close()


def main():
    args = parse()
    if args.windows is None:
        args.windows = 128 if args.workload == "closure" else 256
    if args.workload == "closure":
        if args.impl == "reference":
            run_closure_reference(args)
        else:
            run_closure(args)
        return
    if args.workload in ("window200", "walls200"):
        run_window200(args)
    elif args.workload == "batch":
        if args.impl == "reference":
            run_batch_reference(args)
        else:
            run_batch(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
