"""Row passes whose lines run warp by warp (warp barriers only: split-2 plans,
split-1 plans with A = B, and split-1 plans with B > A, whose row tile keeps B
threads per line in both stages), on batches large enough that many CTAs, and
the warps of one CTA, are in different stages at once.

A line's result cannot depend on what the other lines of its CTA do, so a scan
of 64 positions in 64-wave launches must give, bit for bit, what the same
positions give one at a time (one wave per launch), and what the same batched
scan gives again.  A race between the lines of a CTA (one line's exchange
writing into another line's region) shows up as a difference.  Every row plan
of each length is run, on a specimen whose propagator has the 2/3 band gap (so
warps of dead rows exit early), with readout planes (the readout row pass).
"""
import numpy as np
import pytest

from tests import golden_cases as G
from tests import product_cases as PC

pytestmark = pytest.mark.gpu
GPU = 2
# row plans with warp-local lines: 128 (8x16 pair), 192 (12x16), 240 (15x16),
# 256 (16x16), 512 (16x32 pair), 768 (24x32), 1024 (32x32)
SIZES = [128, 192, 240, 256, 512, 768, 1024]


@pytest.fixture(scope="module")
def J():
    import jmultislicelib_b200 as jb

    return jb.JMS()


def _setup(J, n, nobj=6, nvar=2, ndetper=3):
    a = b = 0.045 * n
    J.cleanup()
    J.set_high_tension(300.0)
    J.set_grid(n, n, a, b, 0.4)
    pro = J.calc_propagator(0.19525, 0.0, 0.0, 1)
    dets = [J.calc_ring_detector(b0, b1) for (b0, b1) in ((0, 10), (20, 50), (60, 150))]
    probe = J.calc_probe(22.0)
    pgr = PC.synthetic_specimen(n, n, 2, nvar, 7 + n)
    objslc = np.arange(nobj) % 2
    assert J.setup(GPU, [nvar, nvar], objslc, [0, 0], ndetper, 3, G.INT) == [0, 0, 0, 0]
    for s in range(2):
        J.set_phase_grating(GPU, s, pgr[s])
    J.set_propagator(GPU, 0, pro)
    for i, (d, m) in enumerate(dets):
        J.set_detector(GPU, i, d, m)
    assert J.init_core(GPU) == 0
    J.set_incident_wave(GPU, probe)
    # the propagator's band gap: the rows the row pass skips
    dead = np.all(np.asarray(pro).reshape(n, -1) == 0, axis=1)
    assert dead.sum() > n // 4, dead.sum()
    return a, b, nobj


@pytest.mark.parametrize("n", SIZES)
def test_batched_rows_equal_single_waves(J, n):
    a, b, nobj = _setup(J, n)
    pos = np.random.default_rng(n).uniform(0, a, (64, 2)).astype(np.float32)
    varseq = np.zeros((1, nobj), np.int32)
    nplan = J.L.JMS_PlanCount(n)
    try:
        for ir in range(nplan):
            assert J.L.JMS_SelectPlans(ir, 0) == 0
            J.L.JMS_SetScanBatch(64)
            e, batched, _ = J.scan(pos, 1, varseq=varseq)
            assert e == 0, e
            e, again, _ = J.scan(pos, 1, varseq=varseq)
            assert e == 0, e
            J.L.JMS_SetScanBatch(1)
            e, single, _ = J.scan(pos, 1, varseq=varseq)
            assert e == 0, e
            assert np.abs(batched).max() > 0
            assert np.array_equal(batched, again), (n, ir)
            assert np.array_equal(batched, single), (n, ir, np.abs(batched - single).max())
    finally:
        J.L.JMS_SetScanBatch(32)
        J.L.JMS_SelectPlans(0, 0)
