"""Parity of the CUDA product (through its C ABI) with the reference and the
FP64 oracle.  The bar: integrated detector signals within 1e-4 relative (per
detector, against the largest value of that detector over the planes), the
same bar for full-size readout arrays (against the array's largest value)."""
import numpy as np
import pytest

from tests import golden_cases as G
from tests import product_cases as PC

pytestmark = pytest.mark.gpu
TOL = 1e-4
GPU = 2


def det_rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.maximum(np.abs(b).max(axis=0), 1e-30)
    return float((np.abs(a - b).max(axis=0) / den).max())


@pytest.fixture(scope="module")
def J():
    import jmultislicelib_b200 as jb

    return jb.JMS()


@pytest.mark.parametrize("name", G.CASES)
def test_golden_case_matches_reference(J, name):
    c, out = PC.run_case(J, name)
    assert out["ndetslc"] == int(c["ndetslc"])
    if "det_int" in c:
        assert det_rel(out["det_int"], c["det_int"]) < TOL
    for key in ("dif", "img", "wff", "wfr", "img_avg", "dif_avg", "wfr_avg", "wff_avg"):
        if key in c:
            assert G.rel_err(out[key], c[key]) < TOL, key
    for key in ("img_avg", "dif_avg", "wfr_avg", "wff_avg"):
        if key in c:
            assert abs(out[key + "_w"] - float(c[key + "_w"])) < 1e-6
    if "rda_int" in c:   # CJMultiSlice::ReadoutDetAvg
        nd = int(c["ndetslc"])
        assert det_rel(out["rda_int"].reshape(nd, -1), c["rda_int"].reshape(nd, -1)) < TOL
        assert abs(out["rda_w"] - float(c["rda_w"])) < 1e-6
    for key in ("rda_img", "rda_dif"):
        if key in c:
            assert G.rel_err(out[key], c[key]) < TOL, key


def test_unscramble_hash_matches_reference(J):
    c, _ = PC.run_case(J, "msa")
    np.testing.assert_array_equal(J.unscramble_hash(), c["unscramble"])


def _oracle_single(J, nx, ny, nobj, ndetper, seed, ntype=1, probe_alpha=22.0, imagedet=G.INT | G.DIF,
                   islc0=0, nvar=2, dx=0.21, dy=0.17, plans=None):
    """Product vs FP64 oracle on a synthetic specimen of any supported size."""
    from oracle import oracle as OR

    a = 0.045 * nx
    b = 0.045 * ny
    J.cleanup()
    wl = J.set_high_tension(300.0)
    J.set_grid(nx, ny, a, b, 0.4)
    pro = J.calc_propagator(0.19525, 0.0, 0.0, ntype)
    dets = [J.calc_ring_detector(b0, b1) for (b0, b1) in ((0, 10), (20, 50), (80, 200))]
    probe = J.calc_probe(probe_alpha, abrr=np.r_[np.zeros(10), 1000.0, np.zeros(37)].astype(np.float32))
    pgr = PC.synthetic_specimen(nx, ny, 2, nvar, seed)
    objslc = np.arange(nobj) % 2
    assert J.setup(GPU, [nvar, nvar], objslc, [0, 0], ndetper, 3, imagedet) == [0, 0, 0, 0]
    for s in range(2):
        assert J.set_phase_grating(GPU, s, pgr[s]) == 0
    assert J.set_propagator(GPU, 0, pro) == 0
    for i, (d, m) in enumerate(dets):
        assert J.set_detector(GPU, i, d, m) == 0
    assert J.init_core(GPU) == 0
    if plans is not None:
        assert J.L.JMS_SelectPlans(*plans) == 0
    assert J.set_incident_wave(GPU, probe) == 0
    J.seed(seed)
    assert J.offset(GPU, dx, dy, 0.0) == 0
    assert J.gpu_multislice(islc0, 0, 1.0) == 0
    nd = J.num_det_planes()
    di = J.get_result(GPU, G.INT, nd * 3).reshape(nd, 3)
    dif = J.get_result(GPU, G.DIF, nd * nx * ny).reshape(nd, ny, nx) if imagedet & G.DIF else None
    # oracle: same variant draws (CRng restated), same inputs
    rng = OR.Rng(seed)
    var = rng.variant_sequence([nvar, nvar], objslc)
    n, hsh = OR.detection_planes(ndetper, nobj)
    assert n == nd
    w0 = OR.offset(probe, a, b, wl, dx, dy, 0.0)
    res = OR.multislice(w0, np.concatenate(pgr), objslc * nvar + var, pro[None], np.zeros(nobj, np.int32), hsh, nd,
                        det=np.stack([d for d, _ in dets]), masks=[m for _, m in dets], imagedet=imagedet,
                        islc0=islc0)
    return di, res["det_int"], dif, res["dif"]


@pytest.mark.parametrize("nx,ny,nobj,ndetper", [
    (256, 256, 24, 8), (512, 512, 20, 5), (384, 720, 6, 3), (1024, 1024, 4, 2), (96, 160, 10, 4),
    (240, 120, 8, 0), (480, 320, 6, 2), (768, 640, 3, 1), (960, 24, 6, 2), (16, 48, 12, 4),
    (180, 180, 10, 4), (192, 192, 10, 4)])
def test_sizes_match_fp64_oracle(J, nx, ny, nobj, ndetper):
    di, odi, dif, odif = _oracle_single(J, nx, ny, nobj, ndetper, seed=nx + ny)
    assert det_rel(di, odi) < TOL
    assert G.rel_err(dif, odif) < TOL


@pytest.mark.parametrize("n", [64, 128, 256, 512, 1024, 2048])
def test_every_fft_plan_matches_fp64_oracle(J, n):
    """Each candidate line plan of a length, on rows and on columns."""
    import jmultislicelib_b200 as jb

    count = jb.lib().JMS_PlanCount(n)
    assert count >= 2
    for i in range(count):
        di, odi, dif, odif = _oracle_single(J, n, n, 6, 3, seed=n + i, plans=(i, count - 1 - i))
        assert det_rel(di, odi) < TOL, i
        assert G.rel_err(dif, odif) < TOL, i


def test_autotune_keeps_results(J):
    import ctypes as C

    di0, odi, _, _ = _oracle_single(J, 512, 512, 8, 4, seed=3)
    ms_r, ms_c = C.c_float(0), C.c_float(0)
    ir, ic = C.c_int(-1), C.c_int(-1)
    assert J.L.JMS_Autotune(4, 3, C.byref(ms_r), C.byref(ms_c), C.byref(ir), C.byref(ic)) == 0
    assert 0 <= ir.value < J.L.JMS_PlanCount(512) and 0 <= ic.value < J.L.JMS_PlanCount(512)
    assert ms_r.value > 0 and ms_c.value > 0
    di1, _, _, _ = _oracle_single(J, 512, 512, 8, 4, seed=3)   # a new setup reuses the tuned plans
    assert det_rel(di1, odi) < TOL
    J.L.JMS_SelectPlans(0, 0)


def test_planar_propagator_and_start_slice(J):
    di, odi, _, _ = _oracle_single(J, 128, 128, 12, 3, seed=5, ntype=0, islc0=5, imagedet=G.INT)
    assert det_rel(di, odi) < TOL


def test_no_object_slices_reads_exit_plane(J):
    # islc0 = nobjslc: only the exit-plane readout of the incoming wave
    di, odi, dif, odif = _oracle_single(J, 64, 64, 6, 2, seed=9, islc0=6)
    assert det_rel(di, odi) < TOL
    assert G.rel_err(dif, odif) < TOL


def test_long_run_512_200_slices(J):
    """The scan workload's depth: 200 slices on 512^2 stays within 1e-4."""
    di, odi, _, _ = _oracle_single(J, 512, 512, 200, 20, seed=31, imagedet=G.INT, nvar=4)
    assert det_rel(di, odi) < TOL


def test_scan_matches_oracle_and_bins(J):
    """Batched scan: positions x phonon passes with explicit variant lists, the
    integrated detectors and the binned, unscrambled exit pattern."""
    from oracle import oracle as OR

    nx = ny = 128
    nobj, nvar, npass, ndetper = 16, 3, 3, 4
    a = b = 0.045 * nx
    J.cleanup()
    wl = J.set_high_tension(300.0)
    J.set_grid(nx, ny, a, b, 0.4)
    pro = J.calc_propagator(0.19525, 0.0, 0.0, 1)
    dets = [J.calc_ring_detector(b0, b1) for (b0, b1) in ((0, 10), (20, 50), (80, 200))]
    probe = J.calc_probe(22.0)
    pgr = PC.synthetic_specimen(nx, ny, 2, nvar, 77)
    objslc = np.arange(nobj) % 2
    assert J.setup(GPU, [nvar, nvar], objslc, [0, 0], ndetper, 3, G.INT) == [0, 0, 0, 0]
    for s in range(2):
        J.set_phase_grating(GPU, s, pgr[s])
    J.set_propagator(GPU, 0, pro)
    for i, (d, m) in enumerate(dets):
        J.set_detector(GPU, i, d, m)
    assert J.init_core(GPU) == 0
    J.set_incident_wave(GPU, probe)
    rng = np.random.default_rng(3)
    pos = rng.uniform(0, a, (7, 2)).astype(np.float32)
    orng = OR.Rng(101)
    varseq = np.stack([orng.variant_sequence([nvar, nvar], objslc) for _ in range(npass)])
    J.L.JMS_SetScanBatch(3)  # 7 positions -> chunks of 3, 3, 1
    e, out, ob = J.scan(pos, npass, varseq=varseq, bin=4)
    assert e == 0
    n, hsh = OR.detection_planes(ndetper, nobj)
    det = np.stack([d for d, _ in dets])
    masks = [m for _, m in dets]
    for ip in range(len(pos)):
        acc = None
        for p in range(npass):
            w0 = OR.offset(probe, a, b, wl, float(pos[ip, 0]), float(pos[ip, 1]))
            acc = OR.multislice(w0, np.concatenate(pgr), objslc * nvar + varseq[p], pro[None],
                                np.zeros(nobj, np.int32), hsh, n, det=det, masks=masks, imagedet=G.INT | G.DIF,
                                weight=1.0 / npass, acc=acc)
        assert det_rel(out[ip], acc["det_int"]) < TOL
        exitdif = np.fft.fftshift(acc["dif"][n - 1])
        binned = exitdif.reshape(ny // 4, 4, nx // 4, 4).sum(axis=(1, 3))
        assert G.rel_err(ob[ip], binned) < TOL
    J.L.JMS_SetScanBatch(32)


def test_descan_shifts_readout(J):
    """Integer-pixel diffraction descan (DescanDifN): the pattern is read out at
    (kx - dnx, ky - dny), and the detectors integrate the shifted pattern."""
    c = G.case("msa")
    PC.setup_case(J, c)
    nx, ny = c["nx"], c["ny"]
    N = nx * ny
    runs = [(0.3, 0.2, 0.0)]

    def run():
        J.seed(c["seed"])
        for dx, dy, dz in runs:
            J.offset(GPU, dx, dy, dz)
            assert J.gpu_multislice(0, 0, 1.0) == 0
        nd = J.num_det_planes()
        return (J.get_result(GPU, G.DIF, nd * N).reshape(nd, ny, nx),
                J.get_result(GPU, G.INT, nd * c["ndet"]).reshape(nd, c["ndet"]))

    dif0, _ = run()
    J.L.DiffractionDescan(1)
    J.L.SetDiffractionDescanN(GPU, 3, -2, 0)
    dif1, di1 = run()
    J.L.DiffractionDescan(0)
    expect = np.roll(dif0, (2, -3), axis=(1, 2))
    assert G.rel_err(dif1, expect) < 1e-6
    det_eff = []
    for d, m in zip(c["det"], c["msk"]):
        if len(m):
            e = np.zeros(N, np.float64)
            np.add.at(e, m, d.ravel()[m])
            det_eff.append(e.reshape(ny, nx))
        else:
            det_eff.append(d.astype(np.float64))
    expect_int = np.einsum("pyx,dyx->pd", expect.astype(np.float64), np.stack(det_eff))
    assert det_rel(di1, expect_int) < 1e-5


def test_scan_with_plasmon_paths(J):
    """Batched scan with the plasmon Monte-Carlo: every wave of every pass
    draws its own path (positions in order, after the pass's variant draw)."""
    from oracle import oracle as OR

    c = G.case("msh")
    PC.setup_case(J, c)
    nx, ny = c["nx"], c["ny"]
    nobj = len(c["objslc"])
    pos = np.array([[0.1, 0.2], [0.5, 0.3], [0.9, 1.1]], np.float32)
    npass = 2
    orng = OR.Rng(5)
    varseq = np.stack([orng.variant_sequence(c["nvar"], c["objslc"]) for _ in range(npass)])
    J.seed(44)
    J.L.JMS_SetScanBatch(2)          # chunks of 2 and 1 waves
    try:
        e, out, _ = J.scan(pos, npass, varseq=varseq)
    finally:
        J.L.JMS_SetScanBatch(32)
        J.L.SetPlasmonMC(0, 0.0, 0.0, 0.0, 0)
    assert e == 0
    qe, qc, mfp, nmax = (float(v) for v in c["plasmon"])
    rng = OR.Rng(44)
    paths = {}
    for p0 in range(0, len(pos), 2):
        for ip in range(npass):
            for iw in range(p0, min(p0 + 2, len(pos))):
                paths[(iw, ip)] = rng.plasmon_shifts(c["slcthick"][c["objslc"]], np.float32(c["a"]),
                                                     np.float32(c["b"]), qe, qc, mfp, int(nmax))
    assert any(paths[k].any() for k in paths)
    n, hsh = OR.detection_planes(c["ndetper"], nobj)
    base = np.concatenate([[0], np.cumsum(c["nvar"])[:-1]]).astype(np.int64)
    for iw in range(len(pos)):
        acc = None
        for ip in range(npass):
            w0 = OR.offset(c["probe"], c["a"], c["b"], c["wl"], float(pos[iw, 0]), float(pos[iw, 1]))
            acc = OR.multislice(w0, np.concatenate(c["pgr"]), (base[c["objslc"]] + varseq[ip]).astype(np.int32),
                                np.stack(c["pro"]), c["proidx"][c["objslc"]], hsh, n, det=np.stack(c["det"]),
                                masks=c["msk"], imagedet=G.INT, weight=1.0 / npass, acc=acc,
                                shifts=paths[(iw, ip)])
        assert det_rel(out[iw], acc["det_int"][:, :c["ndet"]]) < TOL

def test_slice_files_load_into_setup(J, tmp_path):
    """Gratings loaded from EMS slice files (JMS_SliLoadSlice) run exactly as
    the same gratings uploaded with SetSlicePhaseGratings."""
    import jmultislicelib_b200 as jb

    c, ref_out = PC.run_case(J, "msb")
    PC.setup_case(J, c)
    for s, gr in enumerate(c["pgr"]):
        p = str(tmp_path / f"msb_{s + 1:03d}.sli")
        assert jb.sli_write(p, gr, 0.2, c["kv"], c["a"], c["b"]) == 0
        assert J.sli_load_slice(p, s) == 0
    J.seed(c["seed"])
    for (dx, dy, dz, ibtx, ibty, accmode, w) in c["runs"]:
        assert J.offset(GPU, float(dx), float(dy), float(dz), 0, int(ibtx), int(ibty)) == 0
        assert J.gpu_multislice(c["islc0"], int(accmode), float(w)) == 0
    nd = J.num_det_planes()
    di = J.get_result(GPU, G.INT, nd * c["ndet"]).reshape(nd, c["ndet"])
    np.testing.assert_array_equal(di, ref_out["det_int"])
    p = str(tmp_path / "wrong_001.sli")
    assert jb.sli_write(p, np.ones((1, 8, 8), np.complex64), 0.2, 300.0, 1.0, 1.0) == 0
    assert J.sli_load_slice(p, 0) == 7
