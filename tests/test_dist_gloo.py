"""The multi-rank path on CPU: two gloo ranks split a window list round-robin,
step their windows on the oracle and all-reduce the FP64 ledgers; the table
must equal one process stepping every window."""
import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle as O
import silt_scenes as S
import silt_shard

DT = 1.0 / 120.0
N_WIN = 5


def windows():
    return [S.grid(res=r, seed=0x777 + r, puddles=2) for r in (24, 32, 28, 40, 36)][:N_WIN]


def step_windows(idx, wins):
    out = {}
    for w in idx:
        c = O.Core(res=wins[w]["res"], fine_res=64, layout=1)
        S.seed_core(c, wins[w])
        for _ in range(3):
            c.step(DT)
        led = c.ledger()
        out[w] = dict(water_m3=led["water64"], slurry_m3=led["slurry64"], frozen_water_m3=0.0,
                      frozen_slurry_m3=0.0, spray_m3=led["spray_m3"], opened_m3=0.0,
                      total_m3=led["water64"] + led["slurry64"] + led["spray_m3"], cut_m3=0.0, reach_m3=0.0,
                      round_m3=0.0, suspended_m3=0.0, settled_suspended_m3=0.0, frozen_suspended_m3=0.0,
                      entrained_m3=0.0, turbid_m3=0.0, turbid_settled_m3=0.0, frozen_turbid_m3=0.0, stirred_m3=0.0)
    return out


def _rank(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        wins = windows()
        mine = silt_shard.shard(len(wins), rank, world)
        table = silt_shard.gather_ledgers(step_windows(mine, wins), len(wins), dist)
        q.put((rank, mine, table))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_covers_every_window_once():
    for n in (1, 5, 256):
        for world in (1, 2, 3, 8):
            seen = sorted(w for r in range(world) for w in silt_shard.shard(n, r, world))
            assert seen == list(range(n))


def test_two_gloo_ranks_gather_the_single_process_ledgers():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    wins = windows()
    single = silt_shard.gather_ledgers(step_windows(range(len(wins)), wins), len(wins))
    shares = sorted(w for _, mine, _ in got for w in mine)
    assert shares == list(range(len(wins)))
    for _, _, table in got:
        assert np.array_equal(table, single)
