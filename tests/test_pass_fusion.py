"""Frozen-phonon configurations in one launch (JMS_SetPassFusion).

A scan with a variant sequence and fewer positions than the scan batch puts
several configurations of its positions into each launch sequence (wave
k * npos + p = position p in configuration k, each wave reading its own
grating).  Checked on a 128^2 specimen with 2 slice types x 3 variants:
- against the FP64 oracle's multislice of every (position, configuration)
  pair, averaged: integrated detectors and the binned exit pattern within the
  product's 1e-4 bar;
- against the sequential form (one launch sequence per configuration): the
  same waves, so the detector sums agree to FP64 rounding (1e-12) and the
  binned patterns to float atomic-add order (1e-6), with fewer launches;
- with 3 positions and a batch of 8, configurations go 2, 2, 1 per launch
  sequence (an uneven last group).
"""
import numpy as np
import pytest

from tests import golden_cases as G
from tests import product_cases as PC

pytestmark = pytest.mark.gpu
GPU = 2
TOL = 1e-4


@pytest.fixture(scope="module")
def J():
    import jmultislicelib_b200 as jb

    return jb.JMS()


def _setup(J, nx, nobj, nvar, ndetper):
    a = b = 0.045 * nx
    J.cleanup()
    wl = J.set_high_tension(300.0)
    J.set_grid(nx, nx, a, b, 0.4)
    pro = J.calc_propagator(0.19525, 0.0, 0.0, 1)
    dets = [J.calc_ring_detector(b0, b1) for (b0, b1) in ((0, 10), (20, 50), (80, 200))]
    probe = J.calc_probe(22.0)
    pgr = PC.synthetic_specimen(nx, nx, 2, nvar, 91)
    objslc = np.arange(nobj) % 2
    assert J.setup(GPU, [nvar, nvar], objslc, [0, 0], ndetper, 3, G.INT) == [0, 0, 0, 0]
    for s in range(2):
        J.set_phase_grating(GPU, s, pgr[s])
    J.set_propagator(GPU, 0, pro)
    for i, (d, m) in enumerate(dets):
        J.set_detector(GPU, i, d, m)
    assert J.init_core(GPU) == 0
    J.set_incident_wave(GPU, probe)
    return dict(a=a, b=b, wl=wl, pro=pro, dets=dets, probe=probe, pgr=pgr, objslc=objslc)


@pytest.mark.parametrize("batch", [32, 8])
def test_fused_configurations(J, batch):
    from oracle import oracle as OR

    nx, nobj, nvar, npass, ndetper = 128, 16, 3, 5, 4
    st = _setup(J, nx, nobj, nvar, ndetper)
    pos = np.random.default_rng(5).uniform(0, st["a"], (3, 2)).astype(np.float32)
    orng = OR.Rng(202)
    varseq = np.stack([orng.variant_sequence([nvar, nvar], st["objslc"]) for _ in range(npass)]).astype(np.int32)
    J.L.JMS_SetScanBatch(batch)
    res = {}
    for fuse in (1, 0):
        J.L.JMS_SetPassFusion(fuse)
        l0 = J.L.JMS_KernelLaunches()
        e, out, ob = J.scan(pos, npass, varseq=varseq, bin=4)
        assert e == 0, e
        res[fuse] = (out.astype(np.float64), ob.astype(np.float64), J.L.JMS_KernelLaunches() - l0)
    J.L.JMS_SetPassFusion(1)
    J.L.JMS_SetScanBatch(32)
    (fi, fb, fl), (si, sb, sl) = res[1], res[0]
    # the same waves in either form
    assert np.abs(fi - si).max() <= 1e-12 * np.abs(si).max() + 1e-300
    assert np.abs(fb - sb).max() <= 1e-6 * np.abs(sb).max()
    assert fl < sl, (fl, sl)
    # against the FP64 oracle, averaged over the configurations
    n, hsh = OR.detection_planes(ndetper, nobj)
    det = np.stack([d for d, _ in st["dets"]])
    masks = [m for _, m in st["dets"]]
    for ip in range(len(pos)):
        acc = None
        for p in range(npass):
            w0 = OR.offset(st["probe"], st["a"], st["b"], st["wl"], float(pos[ip, 0]), float(pos[ip, 1]))
            acc = OR.multislice(w0, np.concatenate(st["pgr"]), st["objslc"] * nvar + varseq[p], st["pro"][None],
                                np.zeros(nobj, np.int32), hsh, n, det=det, masks=masks, imagedet=G.INT | G.DIF,
                                weight=1.0 / npass, acc=acc)
        den = np.maximum(np.abs(acc["det_int"]).max(axis=0), 1e-30)
        assert (np.abs(fi[ip] - acc["det_int"]).max(axis=0) / den).max() < TOL
        exitdif = np.fft.fftshift(acc["dif"][n - 1])
        binned = exitdif.reshape(nx // 4, 4, nx // 4, 4).sum(axis=(1, 3))
        assert G.rel_err(fb[ip], binned) < TOL
