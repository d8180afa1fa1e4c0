"""The reference's own benchmark driver, JMSBench1, on this library.

oracle/Makefile builds the driver's unmodified sources (test/JMSBench1/*.cpp)
twice: jmsbench1_ref on the reference library, and jmsbench1_b200 with
include/JMultiSlice.h in place of the reference's class header, linked to
libjms_b200.so.  The second binary contains no multislice engine of its own:
every CJMultiSlice method it calls is resolved from libjms_b200.so.  Both run
the same control file and slice files (written by this library's .sli writer)
with every output channel of the driver: annular detectors, per-position
diffraction patterns and probe images, position-averaged ones, and the
elastic / thermal-diffuse separation (test/JMSBench1/multislice.cpp:469-688,
814-997).  The B200 run on the GPU must reproduce the reference's CPU run
(CPUMultislice on MKL) and the reference's own GPU run (cuFFT) file by file.
"""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "jmsbench1_ref")
B200 = os.path.join(ROOT, "oracle", "_ref", "jmsbench1_b200")

needs_bins = pytest.mark.skipif(not (os.access(REF, os.X_OK) and os.access(B200, os.X_OK)),
                                reason="JMSBench1 binaries not built (make -C oracle jmsbench1)")

CONTROL = """set_gpu_id
{gpu}
set_cpu_num
{cpu}
set_sample_input_form
2
set_slc_num
2
set_slc_file_name
'spec'
set_sample_thickness_max
12
set_sample_thickness_step
4
set_sample_tilt
0 0
set_probe_ekv
300.000000
set_probe_convergence
22.000000
set_probe_aberration
6 1000.0 0.0
set_scan_beam_pos
0.4 0.3
set_scan_frame_size
0.6 0.4
set_scan_sampling
3 2
set_scan_frame_rot
30
set_det_annular
0 10 0.0 0.0 BF
set_det_annular
12 24 0.0 0.0 ABF
set_det_annular
30 50 0.0 0.0 ADF
set_det_dif
set_det_padif
set_det_img
set_det_paimg
set_det_separate_tds
set_num_repeat
2
set_output_file
'res'
"""


@needs_bins
def test_b200_driver_takes_the_engine_from_the_library():
    """No CJMultiSlice code inside the driver binary; ldd finds libjms_b200.so."""
    nm = subprocess.run(["nm", "-C", B200], capture_output=True, text=True).stdout
    defined = [ln for ln in nm.splitlines() if "CJMultiSlice::" in ln and " U " not in ln]
    assert not defined, defined[:5]
    assert " U CJMultiSlice::GPUMultislice(int, int, float)" in nm
    ldd = subprocess.run(["ldd", B200], capture_output=True, text=True).stdout
    assert "libjms_b200.so" in ldd and "not found" not in ldd.split("libjms_b200.so")[1].splitlines()[0]


def _specimen(d):
    import jmultislicelib_b200 as jb
    from tests import product_cases as PC

    nx = ny = 64
    a = b = 0.0125 * nx   # 2/3 band limit at 52 mrad (300 kV)
    pgr = PC.synthetic_specimen(nx, ny, 2, 1, 21)
    thick = (0.19525, 0.2)
    # slice 1 has two identical variants: the driver seeds its variant draws
    # from the clock, so distinct variants would make runs differ
    grs = (np.concatenate([pgr[0], pgr[0]]), pgr[1])
    for s in range(2):
        assert jb.sli_write(os.path.join(d, f"spec_{s + 1:03d}.sli"), grs[s], thick[s], 300.0, a, b,
                            title=f"slice {s}") == 0


def _run(exe, d, gpu, cpu):
    os.makedirs(d, exist_ok=True)
    _specimen(d)
    with open(os.path.join(d, "control"), "w") as f:
        f.write(CONTROL.format(gpu=gpu, cpu=cpu))
    r = subprocess.run([exe, "-c", "control", "/silent"], cwd=d, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    out = {f: np.fromfile(os.path.join(d, f), np.float32) for f in os.listdir(d) if f.endswith(".bin")}
    assert out, r.stdout[-2000:] + r.stderr[-2000:]
    return out


def _compare(got, want, what):
    assert sorted(got) == sorted(want), (what, sorted(set(got) ^ set(want)))
    for f, w in want.items():
        g = got[f]
        assert g.shape == w.shape, (what, f)
        # thermal-diffuse files are differences of two channels: bound them by the total
        base = f.replace("_tds", "")
        den = np.abs(want[base] if base in want else w).max()
        err = np.abs(g - w).max() / max(den, 1e-30)
        assert err < 1e-4, (what, f, err)


@pytest.mark.gpu
@needs_bins
def test_reference_driver_on_b200_matches_reference_cpu_and_gpu(tmp_path):
    b200 = _run(B200, str(tmp_path / "b200"), 0, 0)
    ref_cpu = _run(REF, str(tmp_path / "ref_cpu"), -1, 4)
    ref_gpu = _run(REF, str(tmp_path / "ref_gpu"), 0, 0)
    assert any("_ela" in f for f in b200) and "res_padif.bin" in b200 and "res_paimg.bin" in b200
    _compare(b200, ref_cpu, "b200 vs reference CPU")
    _compare(b200, ref_gpu, "b200 vs reference GPU")
