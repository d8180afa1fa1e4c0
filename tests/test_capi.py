"""C-ABI checks that need no GPU: the library loads, exports every declared
symbol, and its host-side generators reproduce the reference bit for bit."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from tests import golden_cases as G

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    txt = open(os.path.join(ROOT, "include", "jms_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    names = re.findall(r"^\s*(?:[A-Za-z_][\w\s\*]*?)\b([A-Za-z_]\w*)\s*\(", txt, flags=re.M)
    return sorted(set(n for n in names if n not in ("if", "while", "return", "sizeof")))


@pytest.fixture(scope="module")
def jb():
    import jmultislicelib_b200 as jb

    jb.lib()
    return jb


def test_library_exports_every_declared_symbol(jb):
    L = C.CDLL(jb.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 60
    for n in names:
        assert hasattr(L, n), n
    assert set(names) == set(jb.SIGNATURES), set(names) ^ set(jb.SIGNATURES)


def test_wavelength_matches_reference(jb):
    g = G.golden()
    J = jb.JMS()
    for kv in (80, 200, 300):
        J.set_high_tension(float(kv))
        assert np.float32(J.L.GetWaveLength()) == g[f"wl_{kv}"]


def test_generators_match_reference_bitwise(jb):
    from tests.golden.make_golden import PROBE_CASES, abrr_array

    g = G.golden()
    J = jb.JMS()
    J.set_high_tension(300.0)
    J.set_grid(64, 48, 1.5, 1.2, 0.39)
    for name, (al, rs, x0, y0, asy, adir, btx, bty, ab) in PROBE_CASES.items():
        np.testing.assert_array_equal(J.calc_probe(al, rs, x0, y0, asy, adir, btx, bty, abrr_array(ab)),
                                      g[f"probe_{name}"])
    for nt in (0, 1):
        np.testing.assert_array_equal(J.calc_propagator(0.19525, 0, 0, nt), g[f"pro_t{nt}"])
        np.testing.assert_array_equal(J.calc_propagator(0.25, 0.5, -0.3, nt), g[f"pro_t{nt}_tilt"])
        for i, (b0, b1, f0, f1, tx, ty, km) in enumerate(g["det_params"]):
            d, m = J.calc_ring_detector(b0, b1, f0, f1, tx, ty, int(km))
            np.testing.assert_array_equal(d, g[f"det_t{nt}_{i}"])
            np.testing.assert_array_equal(m, g[f"msk_t{nt}_{i}"])


def test_probe_is_normalised(jb):
    J = jb.JMS()
    J.set_high_tension(300.0)
    J.set_grid(96, 80, 2.0, 1.7, 0.4)
    w = J.calc_probe(21.0, abrr=np.r_[np.zeros(10), 1200.0, np.zeros(37)].astype(np.float32))
    assert abs((np.abs(w) ** 2).sum() - 1.0) < 1e-5


def test_cpu_code_requests_are_refused(jb):
    """No CPU path in the product: the reference's CPU calls return 1."""
    L = jb.lib()
    n = np.array([1], np.int32)
    ip = n.ctypes.data_as(C.POINTER(C.c_int))
    assert L.PhaseGratingSetup(1, 8, 8, 1, 1, ip) == 1
    assert L.PropagatorSetup(1, 1, ip) == 1
    assert L.DetectorSetup(1, 0, 1, 1, 1) == 1
    assert L.CPUMultislice(0, 0, 1.0, 0) == 1
    assert L.SetIncomingWaveCPU(None, 0, 0) == 1
    assert L.ClearDetMem_h(0) == 1
    assert L.InitCore(1, 1) == 1


def test_unsupported_grid_and_detector_count_are_errors(jb):
    L = jb.lib()
    L.Cleanup()
    L.SetGridSize(1000, 64)
    L.SetSupercellSizeABC(4.0, 4.0, 0.4)
    obj = np.zeros(4, np.int32)
    assert L.ObjectSliceSetup(4, obj.ctypes.data_as(C.POINTER(C.c_int))) == 0
    assert L.InitCore(2, 1) == 103          # 1000 = 2^3 5^3 has no two-factor split <= 32
    assert L.JMS_GridSupported(1000, 64) == 0
    assert L.JMS_GridSupported(720, 384) == 1
    assert L.DetectorSetup(2, 1, 9, 1, 1) == 119   # more than 8 fused integrating detectors
    L.Cleanup()


def test_detector_setup_requires_object_slices(jb):
    L = jb.lib()
    L.Cleanup()
    assert L.DetectorSetup(2, 1, 1, 1, 1) == 101
