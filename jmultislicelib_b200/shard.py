"""Sharding of a STEM scan over ranks (one process per GPU).

Probe positions are independent units of the multislice path (the reference
runs them one by one, test/JMSBench1/multislice.cpp:469-688), so a scan is
split by raster rows over ranks with no exchange during the computation.  The
collectives come at the end: a gather of the small integrated-detector arrays
([npos][ndetslc][ndet] per row) and a sum over ranks of the position-averaged
patterns (the DIFFR_AVG / IMAGE_AVG channels, src/JMultiSlice.h:140-149).
"""
from __future__ import annotations

import numpy as np


def rows_for_rank(nrows: int, rank: int, world: int) -> list[int]:
    """Raster rows handled by `rank`: rank, rank + world, ... (round robin)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank / world size")
    return list(range(rank, nrows, world))


def _to_torch(a: np.ndarray, group):
    import torch
    import torch.distributed as dist

    t = torch.from_numpy(np.array(a, copy=True, order="C"))   # collectives work in place: never on the caller's array
    if dist.get_backend(group) == "nccl":
        t = t.cuda()
    return t


def gather_rows(local: np.ndarray, rows: list[int], nrows: int, group=None) -> np.ndarray:
    """All-gathers per-rank row results into the full scan array.

    local: [len(rows), ...] results of this rank's rows (float or double),
    rows = rows_for_rank(nrows, rank, world); returns [nrows, ...] on every
    rank.  Uses torch.distributed (any backend; device tensors with NCCL).
    """
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    per = -(-nrows // world)                       # rows per rank, padded
    shape = local.shape[1:]
    buf = np.zeros((per,) + shape, local.dtype)
    buf[: len(rows)] = local
    t = _to_torch(buf, group)
    outs = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(outs, t, group=group)
    full = np.zeros((nrows,) + shape, local.dtype)
    for r, o in enumerate(outs):
        rr = rows_for_rank(nrows, r, world)
        full[rr] = o.cpu().numpy()[: len(rr)]
    return full


def allreduce_sum(local: np.ndarray, group=None) -> np.ndarray:
    """Sum of an array over all ranks, returned on every rank: the
    position-averaged diffraction patterns and images of a sharded scan are the
    sums of the ranks' partial sums (divide by the total weight afterwards)."""
    import torch.distributed as dist

    t = _to_torch(local, group)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy()


def check_sharded_scan(scan_row, rank: int, world: int, rows_each: int = 2, group=None):
    """Runs a small sharded scan through both collectives and checks them.

    scan_row(row) -> (integrated [npos, ndetslc, ndet] float64, pattern
    [ny', nx'] float): one raster row of the scan on this rank's device.  The
    scan has rows_each * world rows, split by rows_for_rank.  Returns
    (full integrated [nrows, npos, ndetslc, ndet], summed pattern, report);
    on rank 0 the report compares the gathered rows of the last rank with a
    local rerun of those rows, and the all-reduced pattern with the sum of the
    ranks' gathered partial patterns.  Every rank takes the same collective
    steps in the same order."""
    nrows = rows_each * world
    rows = rows_for_rank(nrows, rank, world)
    res = [scan_row(r) for r in rows]
    local = np.stack([np.asarray(a, np.float64) for a, _ in res])
    pat = np.sum([np.asarray(p, np.float64) for _, p in res], axis=0)
    full = gather_rows(local, rows, nrows, group)
    total = allreduce_sum(pat, group)
    parts = gather_rows(pat[None], [rank], world, group)
    report = {"rows": nrows, "ranks": world}
    if rank == 0:
        last = rows_for_rank(nrows, world - 1, world)
        again = np.stack([np.asarray(scan_row(r)[0], np.float64) for r in last])
        report["rerun_rows"] = last
        report["rerun_max_abs_diff"] = float(np.abs(full[last] - again).max())
        den = max(float(np.abs(total).max()), 1e-300)
        report["pattern_allreduce_rel_diff"] = float(np.abs(total - parts.sum(axis=0)).max() / den)
    return full, total, report
