"""The C++ class interface (include/JMultiSlice.h, JProbeGen.h, rng.h).

A caller written against the reference's CJMultiSlice header
(src/JMultiSlice.h:403-936) compiles against this one and links
libjms_b200.so.  tests/class_api/class_case.cpp is such a caller; it is built
here with g++ and run on golden inputs from the reference:
  - generators through the class, no GPU: bit-identical to the reference;
  - golden multislice cases through the class on the GPU, within 1e-4, and the
    frozen-phonon variant draws of the reference for two seeds, drawn from a
    caller's CRng handed over with SetRng.
The reference's own benchmark driver built on this header is checked in
tests/test_jmsbench1_dropin.py.
"""
import os
import subprocess

import numpy as np
import pytest

from tests import golden_cases as G

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "class_api", "class_case.cpp")
LIBDIR = os.path.join(ROOT, "jmultislicelib_b200")


@pytest.fixture(scope="module")
def app(tmp_path_factory):
    import jmultislicelib_b200 as jb

    jb.lib()
    exe = str(tmp_path_factory.mktemp("class_api") / "class_case")
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-o", exe, SRC, f"-I{ROOT}/include", f"-L{LIBDIR}",
           "-ljms_b200", f"-Wl,-rpath,{LIBDIR}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def _w(d, name, a, dt):
    np.ascontiguousarray(a, dt).tofile(os.path.join(d, name))


def _r(d, name, dt):
    return np.fromfile(os.path.join(d, name), dt)


def test_generators_through_class_match_reference_bitwise(app, tmp_path):
    from tests.golden.make_golden import PROBE_CASES, abrr_array

    g = G.golden()
    d = str(tmp_path)
    gen = [300.0, 64, 48, 1.5, 1.2, 0.39]
    for (al, rs, x0, y0, asy, adir, btx, bty, ab) in PROBE_CASES.values():
        gen += [al, rs, x0, y0, asy, adir, btx, bty] + list(abrr_array(ab))
    for row in g["det_params"]:
        gen += [float(v) for v in row]
    _w(d, "gen.f32", gen, np.float32)
    _w(d, "gen_n.i32", [len(PROBE_CASES), len(g["det_params"])], np.int32)
    r = subprocess.run([app, "gen", d], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, (r.returncode, r.stderr)
    for i, name in enumerate(PROBE_CASES):
        np.testing.assert_array_equal(_r(d, f"probe{i}.c64", np.complex64).reshape(48, 64), g[f"probe_{name}"])
    for nt in (0, 1):
        np.testing.assert_array_equal(_r(d, f"pro_t{nt}.c64", np.complex64).reshape(48, 64), g[f"pro_t{nt}"])
        np.testing.assert_array_equal(_r(d, f"pro_t{nt}_tilt.c64", np.complex64).reshape(48, 64),
                                      g[f"pro_t{nt}_tilt"])
        for i in range(len(g["det_params"])):
            np.testing.assert_array_equal(_r(d, f"det_t{nt}_{i}.f32", np.float32).reshape(48, 64),
                                          g[f"det_t{nt}_{i}"])
            np.testing.assert_array_equal(_r(d, f"msk_t{nt}_{i}.i32", np.int32), g[f"msk_t{nt}_{i}"])
    # CJProbeParams defaults (src/JProbeGen.cpp:53-80) and SetProbeEkV at 300 keV
    dv = _r(d, "probe_defaults.f32", np.float32)
    assert dv[0] == np.float32(0.001969) and dv[1] == np.float32(0.025) and dv[2] == np.float32(0.03)
    assert dv[3] == g["wl_300"]


def test_header_declares_every_public_method_of_the_reference_class():
    """The public methods of src/JMultiSlice.h:403-936, by name."""
    names = """SetDebugLevel Cleanup FreeLibMem SetHighTension SetSupercellSize SetGridSize SetSliceThickness
    SetDetectionPlanes SetPlasmonMC DiffractionDescan SetDiffractionDescanN SetDiffractionDescan
    SetDiffractionDescanMRad CalculateProbeWaveFourier CalculatePropagator CalculateRingDetector PhaseGratingSetup
    ObjectSliceSetup PropagatorSetup DetectorSetup SetPhaseGratingData SetPropagatorData SetDetectorData InitCore
    SetIncidentWave SetIncidentWavePhaseplate ZeroIncidentWavePhaseplate GetUnscrambleHash GetDetetionSliceNum
    GetDetNum GetHighTension GetWaveLength GetGridSize GetSupercellSize GetSliceThickness GetCPUNum GetJCPUcorenum
    GetGPUNum GetGPUName GetCurrentGPU SetCurrentGPU GetGPUStats GetGPUMemInfo SetGPUPgrLoading SetRng GetRng
    SeedRngEx ClearDetMem_h ClearDetMem_d OffsetIncomingWave SetIncomingWaveGPU SetIncomingWaveCPU CPUMultislice
    GPUMultislice GetResult GetAvgResult GetImageAveragingWeight GetWaveAveragingWeight ResetImageAveraging
    ResetWaveAveraging ReadoutDetAvg""".split()
    txt = open(os.path.join(ROOT, "include", "JMultiSlice.h")).read()
    for n in names:
        assert f" {n}(" in txt, n
    out = subprocess.run(["nm", "-DC", os.path.join(LIBDIR, "libjms_b200.so")], capture_output=True,
                         text=True).stdout
    for n in names:
        assert f"CJMultiSlice::{n}(" in out, n


def _write_case(d, c, draws):
    nslc, npro, nobj = len(c["nvar"]), len(c["pro"]), len(c["objslc"])
    _w(d, "cfg.i32", [c["nx"], c["ny"], c["npgx"], c["npgy"], c["ndetper"], c["imagedet"], c["seed"], c["islc0"],
                      c["ndet"], nslc, npro, nobj, len(c["runs"])], np.int32)
    _w(d, "cell.f32", [c["a"], c["b"], c["kv"]], np.float32)
    _w(d, "nvar.i32", c["nvar"], np.int32)
    _w(d, "objslc.i32", c["objslc"], np.int32)
    _w(d, "proidx.i32", c["proidx"], np.int32)
    for s, p in enumerate(c["pgr"]):
        _w(d, f"pgr{s}.c64", p, np.complex64)
    for i, p in enumerate(c["pro"]):
        _w(d, f"pro{i}.c64", p, np.complex64)
    for i in range(c["ndet"]):
        _w(d, f"det{i}.f32", c["det"][i], np.float32)
        _w(d, f"msk{i}.i32", c["msk"][i], np.int32)
    _w(d, "probe.c64", c["probe"], np.complex64)
    if "cppl" in c:
        _w(d, "cppl.f32", c["cppl"], np.float32)
    _w(d, "runs.f32", np.asarray(c["runs"], np.float32).ravel(), np.float32)
    _w(d, "draws_nvar.i32", draws[0], np.int32)
    _w(d, "draws_obj.i32", draws[1], np.int32)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["msa", "mse", "msf"])
def test_golden_case_through_class(app, tmp_path, name):
    g = G.golden()
    c = G.case(name)
    d = str(tmp_path)
    _write_case(d, c, (g["var_nvar"], g["var_objslc"]))
    r = subprocess.run([app, "run", d], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, (r.returncode, r.stderr)
    nd, ndet = (int(v) for v in _r(d, "out_dims.i32", np.int32))
    assert nd == int(c["ndetslc"])
    shp = (nd, c["ny"], c["nx"])
    im = c["imagedet"]
    if im & G.INT:
        got = _r(d, "out_det_int.f32", np.float32).reshape(nd, ndet)
        want = c["det_int"]
        den = np.maximum(np.abs(want).max(axis=0), 1e-30)
        assert (np.abs(got - want).max(axis=0) / den).max() < 1e-4
    for flag, fn, key, dt in ((G.IMG, "out_img.f32", "img", np.float32), (G.DIF, "out_dif.f32", "dif", np.float32),
                              (G.WFR, "out_wfr.c64", "wfr", np.complex64),
                              (G.WFF, "out_wff.c64", "wff", np.complex64)):
        if im & flag:
            assert G.rel_err(_r(d, fn, dt).reshape(shp), c[key]) < 1e-4, key
    if "unscramble" in c:
        np.testing.assert_array_equal(_r(d, "out_unscramble.u32", np.uint32), c["unscramble"].ravel())
    draws = _r(d, "out_draws.i32", np.int32).reshape(2, 3, -1)
    np.testing.assert_array_equal(draws[0], g["var_seed11"])
    np.testing.assert_array_equal(draws[1], g["var_seed12"])
