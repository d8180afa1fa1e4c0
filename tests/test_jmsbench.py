"""The reference-bench-compatible STEM driver (jmultislicelib_b200/jmsbench):
a control file in the reference bench's format, slice files on disk, the
thickness-series images it writes, checked against the FP64 oracle."""
import os
import subprocess

import numpy as np
import pytest

from tests import golden_cases as G
from tests import product_cases as PC

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
APP = os.path.join(ROOT, "jmultislicelib_b200", "jmsbench")

CONTROL = """set_gpu_id
0
set_cpu_num
0
set_sample_input_form
2
set_slc_num
2
set_slc_file_name
'{prefix}'
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
20 50 0.0 0.0 ABF
set_num_repeat
2
set_output_file
'{out}'
"""


def test_driver_is_built():
    assert os.access(APP, os.X_OK)
    r = subprocess.run([APP], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr


def test_driver_rejects_unsupported_commands(tmp_path):
    ctl = tmp_path / "ctl"
    ctl.write_text("set_sample_input_form\n1\nset_structure_file_name\n'x.cel'\n")
    r = subprocess.run([APP, str(ctl)], capture_output=True, text=True)
    assert r.returncode == 1 and "unsupported control command" in r.stderr


@pytest.mark.gpu
def test_driver_scan_matches_oracle(tmp_path):
    import jmultislicelib_b200 as jb
    from oracle import oracle as OR

    nx = ny = 128
    a = b = 0.045 * nx
    thick = (0.19525, 0.2)
    pgr = PC.synthetic_specimen(nx, ny, 2, 1, 21)
    prefix = str(tmp_path / "spec")
    for s in range(2):
        assert jb.sli_write(f"{prefix}_{s + 1:03d}.sli", pgr[s], thick[s], 300.0, a, b, title=f"slice {s}") == 0
    ctl = tmp_path / "control"
    ctl.write_text(CONTROL.format(prefix=prefix, out=str(tmp_path / "res")))
    r = subprocess.run([APP, str(ctl)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    # reference quantities through the library's host generators (bit-identical to the reference)
    J = jb.JMS()
    J.cleanup()
    wl = J.set_high_tension(300.0)
    J.set_grid(nx, ny, a, b, sum(thick))
    pros = [J.calc_propagator(t, 0.0, 0.0, 0) for t in thick]
    dets = [J.calc_ring_detector(b0, b1) for (b0, b1) in ((0, 10), (20, 50))]
    probe = J.calc_probe(22.0, abrr=np.r_[np.zeros(10), 1000.0, np.zeros(37)].astype(np.float32))
    nobj, step = 12, 4
    nd, hsh = OR.detection_planes(step, nobj)
    objslc = np.arange(nobj) % 2
    rot = np.deg2rad(30.0)
    sx, sy = 0.6 / 3, 0.4 / 2
    imgs = {n: np.fromfile(str(tmp_path / f"res_{n}.bin"), np.float32).reshape(nd, 2, 3) for n in ("BF", "ABF")}
    for iy in range(2):
        for ix in range(3):
            dx = 0.4 + np.cos(rot) * sx * ix - np.sin(rot) * sy * iy
            dy = 0.3 + np.cos(rot) * sy * iy + np.sin(rot) * sx * ix
            w0 = OR.offset(probe, a, b, wl, float(np.float32(dx)), float(np.float32(dy)))
            res = OR.multislice(w0, np.concatenate(pgr), objslc, np.stack(pros), objslc, hsh, nd,
                                det=np.stack([d for d, _ in dets]), masks=[m for _, m in dets], imagedet=G.INT)
            for j, n in enumerate(("BF", "ABF")):
                got = imgs[n][:, iy, ix]
                want = res["det_int"][:, j]
                assert np.abs(got - want).max() < 1e-4 * np.abs(want).max(), (n, ix, iy)
