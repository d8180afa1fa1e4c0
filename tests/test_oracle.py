"""Pins the FP64 oracle against the reference's own outputs (CPU, no GPU).

The golden vectors were produced by the reference JMultiSliceLib compiled here
(tests/golden/make_golden.py); the reference runs in FP32 on MKL, so the FP64
oracle must agree to FP32 round-off (tolerances below are far inside the 1e-4
product bar).
"""
import numpy as np
import pytest

from tests import golden_cases as G


def test_fft_matches_numpy():
    from oracle import oracle as OR

    rng = np.random.default_rng(1)
    for ny, nx in ((64, 64), (48, 40), (30, 36), (1, 7), (25, 27), (720 // 8, 384 // 8)):
        z = rng.normal(size=(ny, nx)) + 1j * rng.normal(size=(ny, nx))
        assert G.rel_err(OR.fft2d(z, -1), np.fft.fft2(z)) < 1e-13
        assert G.rel_err(OR.fft2d(z, +1), np.fft.ifft2(z) * nx * ny) < 1e-13


def test_detection_planes_match_reference():
    from oracle import oracle as OR

    g = G.golden()
    for ndetper, nobj in g["planes_list"]:
        n, h = OR.detection_planes(int(ndetper), int(nobj))
        assert n == int(g[f"nplanes_{ndetper}_{nobj}"])
        if nobj > 0:
            np.testing.assert_array_equal(h, g[f"planes_{ndetper}_{nobj}"])


def test_variant_draws_match_reference():
    from oracle import oracle as OR

    g = G.golden()
    for seed in (11, 12):
        rng = OR.Rng(seed)
        seqs = np.stack([rng.variant_sequence(g["var_nvar"], g["var_objslc"]) for _ in range(3)])
        np.testing.assert_array_equal(seqs, g[f"var_seed{seed}"])


@pytest.mark.parametrize("name", G.CASES)
def test_multislice_matches_reference(name):
    c = G.case(name)
    o = G.oracle_case(name)
    assert o["ndetslc"] == int(c["ndetslc"])
    if "det_int" in c:
        assert G.rel_err(o["det_int"][:, : c["ndet"]], c["det_int"]) < 2e-5
    for key in ("dif", "img", "wff", "wfr"):
        if key in c:
            assert G.rel_err(o[key], c[key]) < 2e-5, key
    for key in ("img_avg", "dif_avg", "wfr_avg", "wff_avg"):
        if key in c:
            assert G.rel_err(o["avg"][key[:3]], c[key]) < 2e-5, key
            assert abs(o["avg"]["w"] - float(c[key + "_w"])) < 1e-6


def test_vacuum_propagation_is_defocus():
    """Known answer: with t = 1 everywhere, n Fresnel steps of thickness dz equal
    one multiplication by P(dz)^n (propagators are diagonal in Fourier space),
    and the 1/N of P cancels the unscaled IFT/FT pair of each step."""
    from oracle import oracle as OR

    rng = np.random.default_rng(3)
    ny, nx, n = 32, 48, 5
    wav = (rng.normal(size=(ny, nx)) + 1j * rng.normal(size=(ny, nx))).astype(np.complex64)
    ph = rng.uniform(0, 2 * np.pi, (ny, nx))
    pro = (np.exp(-1j * ph) / (nx * ny)).astype(np.complex64)
    one = np.ones((1, ny, nx), np.complex64)
    _, hsh = OR.detection_planes(0, n)
    res = OR.multislice(wav, one, np.zeros(n, np.int32), pro[None], np.zeros(n, np.int32), hsh, 1, imagedet=0)
    expect = wav.astype(np.complex128) * np.exp(-1j * ph * n)
    assert G.rel_err(res["wave"], expect) < 1e-6  # complex64 input/propagator rounding only


def test_norm_conservation():
    """A pure-phase grating and a unit-modulus propagator conserve sum |psi|^2."""
    from oracle import oracle as OR

    rng = np.random.default_rng(4)
    ny = nx = 32
    wav = np.zeros((ny, nx), np.complex64)
    wav[:4, :4] = 1.0
    wav /= np.sqrt((np.abs(wav) ** 2).sum())
    pgr = np.exp(1j * rng.uniform(0, 2 * np.pi, (2, ny, nx))).astype(np.complex128)
    pro = np.exp(-1j * rng.uniform(0, 2 * np.pi, (ny, nx))) / (nx * ny)
    _, hsh = OR.detection_planes(1, 6)
    det = np.ones((1, ny, nx), np.float32)
    res = OR.multislice(wav, pgr.astype(np.complex64), np.arange(6) % 2, pro.astype(np.complex64)[None],
                        np.zeros(6, np.int32), hsh, 7, det=det, imagedet=1)
    np.testing.assert_allclose(res["det_int"][:, 0], 1.0, rtol=1e-6)


def _det_eff(c):
    """Detector functions with their masks folded in (a masked detector counts
    only its listed pixels; an unmasked one the whole grid)."""
    out = []
    for d, m in zip(c["det"], c["msk"]):
        d = np.asarray(d, np.float64).ravel()
        if len(m):
            e = np.zeros_like(d)
            e[np.asarray(m)] = d[np.asarray(m)]
            d = e
        out.append(d)
    return np.stack(out)


@pytest.mark.parametrize("name", ["msd", "msg"])
def test_readout_det_avg_matches_reference(name):
    """CJMultiSlice::ReadoutDetAvg (src/JMultiSlice.cpp:2667-2945) on the
    oracle's averaged waves: integrated detectors on |<psi(k)>|^2 and the
    |<psi>|^2 patterns."""
    c = G.case(name)
    o = G.oracle_case(name)
    nd = int(c["ndetslc"])
    wff = o["avg"]["wff"].reshape(nd, -1)
    want = (np.abs(wff) ** 2) @ _det_eff(c).T
    assert G.rel_err(c["rda_int"].reshape(nd, -1), want) < 2e-5
    assert abs(float(c["rda_w"]) - o["avg"]["w"]) < 1e-6
    if "rda_img" in c:
        assert G.rel_err(c["rda_img"].reshape(o["avg"]["wfr"].shape), np.abs(o["avg"]["wfr"]) ** 2) < 2e-5
    if "rda_dif" in c:
        assert G.rel_err(c["rda_dif"].reshape(o["avg"]["wff"].shape), np.abs(o["avg"]["wff"]) ** 2) < 2e-5
