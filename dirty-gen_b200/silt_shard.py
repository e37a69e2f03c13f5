"""Windows across ranks (one process per GPU): the window list is split
round-robin and each rank steps its share with no data exchange, since
windows are independent. The one collective is the per-step FP64 ledger
gather: every rank writes its windows' rows, zeros elsewhere, and an
all-reduce SUM gives every rank the full table (each row has one writer, so
the sum is exact)."""
import numpy as np

LEDGER_KEYS = ("water_m3", "slurry_m3", "frozen_water_m3", "frozen_slurry_m3", "spray_m3", "opened_m3", "total_m3",
               "cut_m3", "reach_m3", "round_m3", "suspended_m3", "settled_suspended_m3", "frozen_suspended_m3",
               "entrained_m3", "turbid_m3", "turbid_settled_m3", "frozen_turbid_m3", "stirred_m3")


def shard(n, rank, world):
    """Indices of the windows rank `rank` of `world` steps."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of {world}")
    return list(range(rank, n, world))


def gather_ledgers(local, n, dist=None, device="cpu"):
    """`local`: {window index: ledger dict} of this rank. Returns an n x len(LEDGER_KEYS) FP64
    array (rows in window order, columns LEDGER_KEYS) on every rank."""
    idx = list(local)
    rows = np.array([[float(local[w][k]) for k in LEDGER_KEYS] for w in idx], dtype=np.float64)
    return gather_ledger_rows(idx, rows.reshape(len(idx), len(LEDGER_KEYS)), n, dist, device)


def gather_ledger_rows(windows, rows, n, dist=None, device="cpu"):
    """`rows[k]` (columns LEDGER_KEYS) is window `windows[k]`'s ledger on this
    rank, e.g. `Batch.ledger_rows()`. Returns the n x len(LEDGER_KEYS) FP64 table on every
    rank."""
    import torch

    t = torch.zeros((n, len(LEDGER_KEYS)), dtype=torch.float64)
    if len(windows):
        t[torch.as_tensor(np.asarray(windows, dtype=np.int64))] = torch.from_numpy(np.asarray(rows, np.float64))
    if dist is not None and dist.is_initialized() and dist.get_world_size() > 1:
        t = t.to(device)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.cpu().numpy()
