"""Sharding of a STEM scan over ranks (one process per GPU).

Probe positions are independent units of the multislice path (the reference
runs them one by one, test/JMSBench1/multislice.cpp:469-688), so a scan is
split by raster rows over ranks with no exchange during the computation; the
only collective is the final gather of the small integrated-detector arrays.
"""
from __future__ import annotations

import numpy as np


def rows_for_rank(nrows: int, rank: int, world: int) -> list[int]:
    """Raster rows handled by `rank`: rank, rank + world, ... (round robin)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank / world size")
    return list(range(rank, nrows, world))


def gather_rows(local: np.ndarray, rows: list[int], nrows: int, group=None) -> np.ndarray:
    """All-gathers per-rank row results into the full scan array.

    local: [len(rows), ...] results of this rank's rows (float or double);
    returns [nrows, ...] on every rank.  Uses torch.distributed (any backend).
    """
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    per = -(-nrows // world)                       # rows per rank, padded
    shape = local.shape[1:]
    buf = np.zeros((per,) + shape, local.dtype)
    buf[: len(rows)] = local
    t = torch.from_numpy(buf)
    if dist.get_backend(group) == "nccl":
        t = t.cuda()
    outs = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(outs, t, group=group)
    full = np.zeros((nrows,) + shape, local.dtype)
    for r, o in enumerate(outs):
        rr = rows_for_rank(nrows, r, world)
        full[rr] = o.cpu().numpy()[: len(rr)]
    return full
