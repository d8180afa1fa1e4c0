"""Precision sweep of the FP32 product against the FP64 oracle.

Single probes on 256^2, 512^2, 1024^2 and 2048^2 grids through 200 slices of
strong random-phase gratings (phase 0..3 rad, smoothed by a 0.3 A Gaussian;
jmultislicelib_b200.synthetic.PRECISION_SWEEP).  After 10, 50 and 200
slices the test compares the Fourier-space wave (relative L2 error) and the
three annular detector signals with the oracle's FP64 multislice of the same
inputs.  A detector's error is taken relative to its largest signal over the
planes, or to 1e-3 of the beam intensity where the signal is weaker: the
80-200 mrad signal of these smooth gratings is ~2e-5 of the beam, where the
rounding noise of any FP32 wave (about 1e-7 of the beam per plane) is already
a 1e-3 share.  With JMS_SWEEP_OUT set, the measured errors are appended to that
file as JSON lines.
"""
import json
import os

import numpy as np
import pytest

from tests import golden_cases as G

pytestmark = pytest.mark.gpu
GPU = 2
DET_TOL = 1e-4      # integrated detector signals, relative to max(signal, DET_FLOOR)
DET_FLOOR = 1e-3    # of the beam intensity: weaker signals are held to 1e-7 absolute
WAVE_TOL = 1e-4     # relative L2 of the wave


@pytest.fixture(scope="module")
def J():
    import jmultislicelib_b200 as jb

    return jb.JMS()


def _run(J, n):
    from jmultislicelib_b200 import synthetic as S
    from oracle import oracle as OR

    cfg = S.PRECISION_SWEEP
    a = b = n * cfg["pixel"]
    nobj, ndetper = cfg["nobj"], cfg["ndetper"]
    pgr = S.random_phase_gratings(n, n, a, b, 2, cfg["seed"] + n)
    J.cleanup()
    wl = J.set_high_tension(cfg["kv"])
    J.set_grid(n, n, a, b, S.DZ_SLICE)
    pro = J.calc_propagator(S.DZ_SLICE, 0.0, 0.0, cfg["ntype"])
    dets = [J.calc_ring_detector(b0, b1) for (b0, b1) in cfg["dets"]]
    probe = J.calc_probe(cfg["alpha"])
    objslc = np.arange(nobj) % 2
    flags = G.INT | G.WFF
    assert J.setup(GPU, [1, 1], objslc, [0, 0], ndetper, 3, flags) == [0, 0, 0, 0]
    for s in range(2):
        assert J.set_phase_grating(GPU, s, pgr[s:s + 1]) == 0
    assert J.set_propagator(GPU, 0, pro) == 0
    for i, (d, m) in enumerate(dets):
        assert J.set_detector(GPU, i, d, m) == 0
    assert J.init_core(GPU) == 0
    assert J.set_incident_wave(GPU, probe) == 0
    dx, dy = 0.5 * a, 0.5 * b
    assert J.offset(GPU, dx, dy, 0.0) == 0
    assert J.gpu_multislice(0, 0, 1.0) == 0
    nd = J.num_det_planes()
    di = J.get_result(GPU, G.INT, nd * 3).reshape(nd, 3)
    wff = J.get_result(GPU, G.WFF, nd * n * n, np.complex64).reshape(nd, n, n)
    J.cleanup()

    npl, hsh = OR.detection_planes(ndetper, nobj)
    assert npl == nd
    w0 = OR.offset(probe, a, b, wl, dx, dy, 0.0)
    res = OR.multislice(w0, pgr, objslc, pro[None], np.zeros(nobj, np.int32), hsh, nd,
                        det=np.stack([d for d, _ in dets]), masks=[m for _, m in dets], imagedet=flags)
    odi, owff = res["det_int"], res["wff"]
    rows = []
    for t in cfg["thicknesses"]:
        p = t // ndetper
        dw = np.linalg.norm((wff[p].astype(np.complex128) - owff[p]).ravel()) / np.linalg.norm(owff[p].ravel())
        big = np.abs(odi).max(axis=0)
        dd = np.abs(di[p] - odi[p]) / np.maximum(big, 1e-30)
        dg = np.abs(di[p] - odi[p]) / np.maximum(big, DET_FLOOR)
        rows.append({"n": n, "slices": t, "wave_rel_l2": float(dw), "det_rel": [float(x) for x in dd],
                     "det_rel_floored": [float(x) for x in dg], "det": [float(x) for x in odi[p]]})
    return rows


@pytest.mark.parametrize("n", [256, 512, 1024, 2048])
def test_precision_sweep_fp32(J, n):
    rows = _run(J, n)
    out = os.environ.get("JMS_SWEEP_OUT")
    if out:
        with open(out, "a") as f:
            for r in rows:
                f.write(json.dumps({"form": "fp32", **r}) + "\n")
    for r in rows:
        assert max(r["det_rel_floored"]) < DET_TOL, r
        assert r["wave_rel_l2"] < WAVE_TOL, r
