"""Multi-rank scan sharding on CPU (gloo, world size 2): the row split covers
every raster row exactly once, the gather rebuilds the full scan, and the
all-reduce sums the position-averaged patterns.  The ranks' rows are real
multislice results shaped like JMS_ScanGPU output ([npos][ndetslc][ndet],
float64): each rank runs the FP64 oracle on a small specimen, the way each GPU
runs the library on its rows."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from jmultislicelib_b200 import shard

NROWS_EACH, NPOS = 2, 3


def test_rows_partition_the_raster():
    for nrows in (1, 7, 64):
        for world in (1, 2, 3, 8):
            seen = sorted(r for rank in range(world) for r in shard.rows_for_rank(nrows, rank, world))
            assert seen == list(range(nrows))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _scan_row(row):
    """One raster row: NPOS probe positions through 8 slices of a 32^2 random
    phase object, FP64 oracle; returns (integrated detectors [NPOS, ndetslc, 2],
    sum over the row's positions of the exit-plane diffraction pattern)."""
    from oracle import oracle as OR

    n, a = 32, 1.2
    rng = np.random.default_rng(7)
    pgr = np.exp(1j * rng.uniform(0, 0.6, (2, n, n))).astype(np.complex64)
    k = np.fft.fftfreq(n, d=a / n)
    k2 = k[None, :] ** 2 + k[:, None] ** 2
    probe = (k2 < 8.0 ** 2).astype(np.complex64)
    probe /= np.sqrt((np.abs(probe) ** 2).sum())
    pro = (np.exp(-1j * np.pi * 0.00197 * 0.2 * k2) * (k2 < 12.0 ** 2) / (n * n)).astype(np.complex64)
    dets = np.stack([(k2 < 4.0 ** 2), (k2 >= 5.0 ** 2) & (k2 < 10.0 ** 2)]).astype(np.float32)
    nobj = 8
    nd, hsh = OR.detection_planes(4, nobj)
    objslc = np.arange(nobj) % 2
    out, pat = [], np.zeros((n, n))
    for i in range(NPOS):
        w0 = OR.offset(probe, a, a, 0.00197, 0.1 * i, 0.15 * row)
        res = OR.multislice(w0, pgr, objslc.astype(np.int32), pro[None], np.zeros(nobj, np.int32), hsh, nd,
                            det=dets, masks=[np.zeros(0, np.int32)] * 2, imagedet=1 | 4)
        out.append(res["det_int"])
        pat += res["dif"][-1]
    return np.stack(out), pat


def _worker(rank, world, port, q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        full, total, rep = shard.check_sharded_scan(_scan_row, rank, world, rows_each=NROWS_EACH)
        q.put((rank, full, total, rep))
    finally:
        dist.destroy_process_group()


def test_sharded_scan_gathers_rows_and_sums_patterns_with_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    world = 2
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(world):
        r, full, total, rep = q.get(timeout=300)
        res[r] = (full, total, rep)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    nrows = NROWS_EACH * world
    single = [_scan_row(r) for r in range(nrows)]
    want = np.stack([a for a, _ in single])
    want_pat = np.sum([p for _, p in single], axis=0)
    for r in range(world):
        full, total, _ = res[r]
        assert full.shape == (nrows, NPOS) + want.shape[2:] and full.dtype == np.float64
        np.testing.assert_array_equal(full, want)
        np.testing.assert_allclose(total, want_pat, rtol=1e-12, atol=0)
    rep = res[0][2]
    assert rep["rerun_max_abs_diff"] == 0.0 and rep["pattern_allreduce_rel_diff"] < 1e-12
