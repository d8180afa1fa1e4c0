"""The reference's CPU-runnable case: one probe on a 256^2 grid (3x3 ABO3 cells,
2 slice types, 100 slices, 300 kV, 25 mrad, aberration free, probe at the cell
centre, 0-10 / 20-50 / 80-200 mrad detectors read every 10 slices; the
workload jmultislicelib_b200.synthetic.POINT_256).

CPU: the reference's own CPUMultislice (oracle/_ref, MKL) and the FP64 oracle
agree on it, which pins the oracle on this workload.  GPU: the product's
GPUMultislice matches the FP64 oracle there, on every detector (relative to
max(largest signal, 1e-3 of the beam), the floored criterion of the other
parity tests) and on the exit-plane diffraction pattern.
"""
import os

import numpy as np
import pytest

TOL = 1e-4
FLOOR = 1e-3
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _inputs():
    import jmultislicelib_b200 as jb
    from jmultislicelib_b200 import synthetic as S

    cfg = S.POINT_256
    sp = S.make_specimen(cfg["nx"], cfg["ny"], cfg["ncell"], cfg["ncell"], cfg["nslice_types"], cfg["nvar"],
                         cfg["seed"], cfg["kv"])
    J = jb.JMS()
    J.cleanup()
    wl = J.set_high_tension(cfg["kv"])
    J.set_grid(cfg["nx"], cfg["ny"], sp.a, sp.b, S.DZ_SLICE)
    pro = J.calc_propagator(S.DZ_SLICE, 0.0, 0.0, cfg["ntype"])
    dets = [J.calc_ring_detector(b0, b1) for (b0, b1) in cfg["dets"]]
    probe = J.calc_probe(cfg["alpha"])
    return cfg, sp, J, wl, pro, dets, probe


def _oracle(cfg, sp, wl, pro, dets, probe, pos):
    from oracle import oracle as OR

    nobj = cfg["nobj"]
    objslc = np.arange(nobj) % cfg["nslice_types"]
    nd, hsh = OR.detection_planes(cfg["ndetper"], nobj)
    w0 = OR.offset(probe, sp.a, sp.b, wl, float(pos[0]), float(pos[1]))
    return OR.multislice(w0, np.concatenate(sp.gratings), objslc.astype(np.int32), pro[None],
                         np.zeros(nobj, np.int32), hsh, nd, det=np.stack([d for d, _ in dets]),
                         masks=[m for _, m in dets], imagedet=1 | 4)


def _floored(got, want):
    den = np.maximum(np.abs(want).max(axis=0), FLOOR)
    return np.abs(got - want).max(axis=0) / den


def test_reference_cpu_path_matches_fp64_oracle():
    from oracle import ref

    if not ref.available():
        pytest.skip("oracle/_ref not built")
    cfg, sp, J, wl, pro, dets, probe = _inputs()
    pos = np.array([0.5 * sp.a, 0.5 * sp.b], np.float32)
    want = _oracle(cfg, sp, wl, pro, dets, probe, pos)["det_int"]
    R = ref.RefJMS()
    try:
        R.set_high_tension(cfg["kv"])
        R.set_grid(cfg["nx"], cfg["ny"], sp.a, sp.b, 0.19525)
        nobj = cfg["nobj"]
        R.setup(ref.CODE_CPU, [1] * cfg["nslice_types"], np.arange(nobj) % cfg["nslice_types"],
                [0] * cfg["nslice_types"], cfg["ndetper"], len(dets), 1, 1)
        for s, gr in enumerate(sp.gratings):
            R.set_phase_grating(ref.CODE_CPU, s, gr)
        R.set_propagator(ref.CODE_CPU, 0, pro)
        for i, (d, m) in enumerate(dets):
            R.set_detector(ref.CODE_CPU, i, d, m)
        R.init_core(ref.CODE_CPU, 1)
        R.set_incident_wave(ref.CODE_CPU, probe)
        R.offset(ref.CODE_CPU, float(pos[0]), float(pos[1]), 0.0)
        R.cpu_multislice(0, 0, 1.0, 0)
        got = R.get_result(ref.CODE_CPU, 1, want.size).reshape(want.shape)
    finally:
        R.close()
    assert _floored(got, want).max() < TOL, _floored(got, want)


@pytest.mark.gpu
def test_product_matches_fp64_oracle():
    cfg, sp, J, wl, pro, dets, probe = _inputs()
    pos = np.array([0.5 * sp.a, 0.5 * sp.b], np.float32)
    res = _oracle(cfg, sp, wl, pro, dets, probe, pos)
    objslc = np.arange(cfg["nobj"]) % cfg["nslice_types"]
    assert J.setup(2, [1] * cfg["nslice_types"], objslc, [0] * cfg["nslice_types"], cfg["ndetper"], len(dets),
                   1 | 4) == [0, 0, 0, 0]
    for s, gr in enumerate(sp.gratings):
        assert J.set_phase_grating(2, s, gr) == 0
    assert J.set_propagator(2, 0, pro) == 0
    for i, (d, m) in enumerate(dets):
        assert J.set_detector(2, i, d, m) == 0
    assert J.init_core(2) == 0
    assert J.set_incident_wave(2, probe) == 0
    assert J.offset(2, float(pos[0]), float(pos[1]), 0.0) == 0
    assert J.gpu_multislice(0, 0, 1.0) == 0
    nd = J.num_det_planes()
    di = J.get_result(2, 1, nd * len(dets)).reshape(nd, len(dets))
    err = _floored(di, res["det_int"])
    assert err.max() < TOL, err
    # the two detectors with signal meet the bar relative to their own signal too
    rel = np.abs(di - res["det_int"]).max(axis=0) / np.abs(res["det_int"]).max(axis=0)
    assert rel[:2].max() < TOL, rel
    dif = J.get_result(2, 4, nd * cfg["nx"] * cfg["ny"]).reshape(nd, cfg["ny"], cfg["nx"])
    assert np.abs(dif[-1] - res["dif"][-1]).max() < TOL * np.abs(res["dif"][-1]).max()
