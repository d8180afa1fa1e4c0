"""Multi-rank scan sharding on CPU (gloo, world size 2): the row split covers
every raster row exactly once, and the gather rebuilds the full scan."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from jmultislicelib_b200 import shard


def test_rows_partition_the_raster():
    for nrows in (1, 7, 64):
        for world in (1, 2, 3, 8):
            seen = sorted(r for rank in range(world) for r in shard.rows_for_rank(nrows, rank, world))
            assert seen == list(range(nrows))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, nrows, q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rows = shard.rows_for_rank(nrows, rank, world)
        # stand-in for per-row detector results: [row, plane, detector]
        local = np.stack([np.full((3, 2), 10.0 * r + rank, np.float64) for r in rows])
        full = shard.gather_rows(local, rows, nrows)
        q.put((rank, full))
    finally:
        dist.destroy_process_group()


def test_gather_rebuilds_scan_with_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    nrows, world = 7, 2
    procs = [ctx.Process(target=_worker, args=(r, world, port, nrows, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(world):
        full = res[r]
        for row in range(nrows):
            owner = row % world
            np.testing.assert_array_equal(full[row], np.full((3, 2), 10.0 * row + owner))
