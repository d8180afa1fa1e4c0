"""Tensor-core passes (JMS_SetPrecision 1 = BF16 hi+lo, 2 = FP16 hi+lo) against
the FP64 oracle and against the FP32 passes.

Precision sweep: single probes on 256^2, 512^2, 1024^2 and 2048^2 grids through 200
slices of strong random-phase gratings (jmultislicelib_b200.synthetic
PRECISION_SWEEP, the workload of test_precision_sweep.py), errors after 10,
50 and 200 slices: relative L2 of the Fourier-space wave and the three annular
detector signals relative to max(signal, 1e-3 of the beam).  Readout slices
(every 10th) run the FP32 passes, the other 90 % the tensor-core passes.
With JMS_SWEEP_OUT set, the errors are appended to that file as JSON lines.

Bars: both forms are held to 1e-4 on waves and detectors through 50 slices,
and after 200 slices to 2.5e-4 up to 1024^2 and 4e-4 at 2048^2.  Measured on
a B200 (200 slices, wave / worst detector): FP16 (8 + 11 bits) 4.7e-5 /
8.4e-5 at 256^2, 6.8e-5 / 1.3e-4 at 512^2, 9.8e-5 / 1.7e-4 at 1024^2,
1.4e-4 / 2.5e-4 at 2048^2; BF16 (8 + 8 bits) 7.8e-5 / 6.4e-5, 8.6e-5 /
1.0e-4, 1.05e-4 / 1.4e-4, 1.4e-4 / 2.2e-4; the FP32 passes 2-3e-5 / 4-6e-5.
The tensor-core error grows linearly with thickness: the FP32 accumulation
inside the MMA rounds with a bias, and the main product's K / 16 accumulation
steps per radix stage add it up over the slices (2 + 2 steps per transform
at 256^2, 4 + 4 at 1024^2, 8 + 4 at 2048^2 with its 64-point stage).
"""
import json
import os

import numpy as np
import pytest

from tests import golden_cases as G
from tests.test_precision_sweep import DET_FLOOR

pytestmark = pytest.mark.gpu
GPU = 2
BAR_200 = {256: 2.5e-4, 512: 2.5e-4, 1024: 2.5e-4, 2048: 4e-4}   # after 200 slices
BAR_50 = 1e-4                             # through 50 slices
MODE = {"fp32": 0, "bf16": 1, "fp16": 2}


@pytest.fixture(scope="module")
def J():
    import jmultislicelib_b200 as jb

    return jb.JMS()


def _setup(J, n, nobj, ndetper, flags, seed_off=0):
    from jmultislicelib_b200 import synthetic as S

    cfg = S.PRECISION_SWEEP
    a = b = n * cfg["pixel"]
    pgr = S.random_phase_gratings(n, n, a, b, 2, cfg["seed"] + n + seed_off)
    J.cleanup()
    wl = J.set_high_tension(cfg["kv"])
    J.set_grid(n, n, a, b, S.DZ_SLICE)
    pro = J.calc_propagator(S.DZ_SLICE, 0.0, 0.0, cfg["ntype"])
    dets = [J.calc_ring_detector(b0, b1) for (b0, b1) in cfg["dets"]]
    probe = J.calc_probe(cfg["alpha"])
    objslc = np.arange(nobj) % 2
    assert J.setup(GPU, [1, 1], objslc, [0, 0], ndetper, 3, flags) == [0, 0, 0, 0]
    for s in range(2):
        assert J.set_phase_grating(GPU, s, pgr[s:s + 1]) == 0
    assert J.set_propagator(GPU, 0, pro) == 0
    for i, (d, m) in enumerate(dets):
        assert J.set_detector(GPU, i, d, m) == 0
    assert J.init_core(GPU) == 0
    assert J.set_incident_wave(GPU, probe) == 0
    return dict(a=a, b=b, wl=wl, pgr=pgr, pro=pro, dets=dets, probe=probe, objslc=objslc)


def _run(J, n, form):
    from jmultislicelib_b200 import synthetic as S
    from oracle import oracle as OR

    cfg = S.PRECISION_SWEEP
    nobj, ndetper = cfg["nobj"], cfg["ndetper"]
    flags = G.INT | G.WFF
    st = _setup(J, n, nobj, ndetper, flags)
    assert J.set_precision(MODE[form]) == 0
    tc0 = J.L.JMS_TcLaunches()
    dx, dy = 0.5 * st["a"], 0.5 * st["b"]
    assert J.offset(GPU, dx, dy, 0.0) == 0
    assert J.gpu_multislice(0, 0, 1.0) == 0
    nd = J.num_det_planes()
    di = J.get_result(GPU, G.INT, nd * 3).reshape(nd, 3)
    wff = J.get_result(GPU, G.WFF, nd * n * n, np.complex64).reshape(nd, n, n)
    ntc = J.L.JMS_TcLaunches() - tc0
    status = J.tc_status()
    J.set_precision(0)
    J.cleanup()
    npl, hsh = OR.detection_planes(ndetper, nobj)
    w0 = OR.offset(st["probe"], st["a"], st["b"], st["wl"], dx, dy, 0.0)
    res = OR.multislice(w0, st["pgr"], st["objslc"], st["pro"][None], np.zeros(nobj, np.int32), hsh, nd,
                        det=np.stack([d for d, _ in st["dets"]]), masks=[m for _, m in st["dets"]], imagedet=flags)
    odi, owff = res["det_int"], res["wff"]
    rows = []
    for t in cfg["thicknesses"]:
        p = t // ndetper
        dw = np.linalg.norm((wff[p].astype(np.complex128) - owff[p]).ravel()) / np.linalg.norm(owff[p].ravel())
        big = np.abs(odi).max(axis=0)
        dg = np.abs(di[p] - odi[p]) / np.maximum(big, DET_FLOOR)
        rows.append({"form": form, "n": n, "slices": t, "wave_rel_l2": float(dw),
                     "det_rel_floored": [float(x) for x in dg]})
    return rows, ntc, status


@pytest.mark.parametrize("form", ["fp16", "bf16"])
@pytest.mark.parametrize("n", [256, 512, 1024, 2048])
def test_tc_precision_sweep(J, n, form):
    rows, ntc, status = _run(J, n, form)
    out = os.environ.get("JMS_SWEEP_OUT")
    if out:
        with open(out, "a") as f:
            for r in rows:
                f.write(json.dumps(r) + "\n")
    print(json.dumps(rows))
    assert status == 0
    # 200 slices: every column pass (no image readout here) and the 180 row
    # passes without Fourier readout run on the tensor cores
    assert ntc == 380, ntc
    for r in rows:
        bar = BAR_50 if r["slices"] <= 50 else BAR_200[n]
        assert max(r["det_rel_floored"]) < bar, r
        assert r["wave_rel_l2"] < bar, r


@pytest.mark.parametrize("form", ["fp16", "bf16"])
@pytest.mark.parametrize("n", [256, 512, 1024, 2048])
def test_tc_scan_matches_fp32(J, n, form):
    """Batched scan (JMS_ScanGPU, many waves per launch, band pruning, binned
    exit pattern) with the tensor-core passes against the FP32 passes on the
    same variant draws (40 slices): integrated signals within 1e-4 of the
    largest signal per detector, binned patterns within 1e-4 of their maximum."""
    nobj, ndetper = 40, 10
    _setup(J, n, nobj, ndetper, G.INT, seed_off=7)
    rng = np.random.default_rng(n)
    npos = 24
    a = b = n * 0.0458 / 10.0
    pos = np.stack([rng.uniform(0, a, npos), rng.uniform(0, b, npos)], axis=1).astype(np.float32)
    varseq = np.zeros((2, nobj), np.int32)
    outs = {}
    for f in ("fp32", form):
        assert J.set_precision(MODE[f]) == 0
        e, di, db = J.scan(pos, 2, varseq=varseq, bin=4)
        assert e == 0, e
        outs[f] = (di, db)
    assert J.tc_status() == 0
    J.set_precision(0)
    J.cleanup()
    (i0, b0), (i1, b1) = outs["fp32"], outs[form]
    den = np.maximum(np.abs(i0).max(axis=(0, 1)), 1e-30)
    e_int = float((np.abs(i1 - i0).max(axis=(0, 1)) / den).max())
    e_bin = float(np.abs(b1 - b0).max() / np.abs(b0).max())
    print(n, form, e_int, e_bin)
    assert e_int < BAR_50 and e_bin < BAR_50, (e_int, e_bin)


def test_tc_falls_back_on_unsupported_grid(J):
    """Grid lengths without a tensor-core plan (here 384) keep the FP32 passes:
    the results equal the FP32 mode's bit for bit and no tensor-core pass runs."""
    res = {}
    for f in ("fp32", "fp16"):
        n = 384
        st = _setup(J, n, 20, 10, G.INT)
        assert J.set_precision(MODE[f]) == 0
        tc0 = J.L.JMS_TcLaunches()
        assert J.offset(GPU, 0.5 * st["a"], 0.5 * st["b"], 0.0) == 0
        assert J.gpu_multislice(0, 0, 1.0) == 0
        nd = J.num_det_planes()
        res[f] = (J.get_result(GPU, G.INT, nd * 3), J.L.JMS_TcLaunches() - tc0)
        J.set_precision(0)
    assert res["fp16"][1] == 0
    assert np.array_equal(res["fp32"][0], res["fp16"][0])


@pytest.mark.parametrize("nx,ny", [(512, 256), (256, 1024)])
def test_tc_non_square_grid_matches_fp32(J, nx, ny):
    """Non-square grids: the row pass tiles rows of length nx, the column pass
    columns of length ny, each with its own twiddles and plan.  The BF16
    tensor-core scan matches the FP32 scan within 1e-4 (integrated signals per
    detector, binned patterns of their maximum)."""
    from jmultislicelib_b200 import synthetic as S

    cfg = S.PRECISION_SWEEP
    a, b = nx * cfg["pixel"], ny * cfg["pixel"]
    pgr = np.stack([S.random_phase_gratings(nx, ny, a, b, 1, cfg["seed"] + 11 + k)[0] for k in range(2)])
    nobj = 30
    J.cleanup()
    J.set_high_tension(cfg["kv"])
    J.set_grid(nx, ny, a, b, S.DZ_SLICE)
    pro = J.calc_propagator(S.DZ_SLICE, 0.0, 0.0, cfg["ntype"])
    dets = [J.calc_ring_detector(b0, b1) for (b0, b1) in cfg["dets"]]
    probe = J.calc_probe(cfg["alpha"])
    objslc = np.arange(nobj) % 2
    assert J.setup(GPU, [1, 1], objslc, [0, 0], 10, 3, G.INT) == [0, 0, 0, 0]
    for s_ in range(2):
        assert J.set_phase_grating(GPU, s_, pgr[s_:s_ + 1]) == 0
    assert J.set_propagator(GPU, 0, pro) == 0
    for i, (d, m) in enumerate(dets):
        assert J.set_detector(GPU, i, d, m) == 0
    assert J.init_core(GPU) == 0
    assert J.set_incident_wave(GPU, probe) == 0
    rng = np.random.default_rng(nx + ny)
    pos = np.stack([rng.uniform(0, a, 12), rng.uniform(0, b, 12)], axis=1).astype(np.float32)
    varseq = np.zeros((2, nobj), np.int32)
    outs = {}
    for f in ("fp32", "bf16"):
        assert J.set_precision(MODE[f]) == 0
        tc0 = J.L.JMS_TcLaunches()
        e, di, db = J.scan(pos, 2, varseq=varseq, bin=4)
        assert e == 0, e
        outs[f] = (di, db, J.L.JMS_TcLaunches() - tc0)
    assert J.tc_status() == 0
    J.set_precision(0)
    J.cleanup()
    (i0, b0, _), (i1, b1, ntc) = outs["fp32"], outs["bf16"]
    assert ntc > 0
    den = np.maximum(np.abs(i0).max(axis=(0, 1)), 1e-30)
    e_int = float((np.abs(i1 - i0).max(axis=(0, 1)) / den).max())
    e_bin = float(np.abs(b1 - b0).max() / np.abs(b0).max())
    assert e_int < BAR_50 and e_bin < BAR_50, (e_int, e_bin)

