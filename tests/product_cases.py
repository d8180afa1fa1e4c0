"""Runs golden cases and synthetic cases through the product's C ABI."""
from __future__ import annotations

import numpy as np

from tests import golden_cases as G

GPU = 2


def setup_case(J, c):
    """Loads a golden case's inputs into the library (reference setup chain)."""
    J.cleanup()
    J.set_high_tension(c["kv"])
    J.set_grid(c["nx"], c["ny"], c["a"], c["b"], 0.4)
    e = J.setup(GPU, c["nvar"], c["objslc"], c["proidx"], c["ndetper"], c["ndet"], c["imagedet"],
                npg=(c["npgx"], c["npgy"]))
    assert e == [0, 0, 0, 0], e
    for s, gr in enumerate(c["pgr"]):
        assert J.set_phase_grating(GPU, s, gr) == 0
    for i, p in enumerate(c["pro"]):
        assert J.set_propagator(GPU, i, p) == 0
    for i, (d, m) in enumerate(zip(c["det"], c["msk"])):
        assert J.set_detector(GPU, i, d, m) == 0
    assert J.init_core(GPU) == 0
    assert J.set_incident_wave(GPU, c["probe"]) == 0
    if "cppl" in c:
        assert J.set_phaseplate(GPU, c["cppl"]) == 0
    if "plasmon" in c:
        for s_, t_ in enumerate(c["slcthick"]):
            J.L.SetSliceThickness(s_, float(t_))
        qe, qc, mfp, nmax = (float(v) for v in c["plasmon"])
        J.L.SetPlasmonMC(1, qe, qc, mfp, int(nmax))
    else:
        J.L.SetPlasmonMC(0, 0.0, 0.0, 0.0, 0)


def run_case(J, name):
    c = G.case(name)
    setup_case(J, c)
    J.seed(c["seed"])
    for (dx, dy, dz, ibtx, ibty, accmode, w) in c["runs"]:
        assert J.offset(GPU, float(dx), float(dy), float(dz), 0, int(ibtx), int(ibty)) == 0
        e = J.gpu_multislice(c["islc0"], int(accmode), float(w))
        assert e == 0, e
    nd = J.num_det_planes()
    N = c["nx"] * c["ny"]
    shp = (nd, c["ny"], c["nx"])
    out = {"ndetslc": nd}
    im = c["imagedet"]
    if im & G.INT:
        out["det_int"] = J.get_result(GPU, G.INT, nd * c["ndet"]).reshape(nd, c["ndet"])
    if im & G.DIF:
        out["dif"] = J.get_result(GPU, G.DIF, nd * N).reshape(shp)
    if im & G.IMG:
        out["img"] = J.get_result(GPU, G.IMG, nd * N).reshape(shp)
    if im & G.WFF:
        out["wff"] = J.get_result(GPU, G.WFF, nd * N, np.complex64).reshape(shp)
    if im & G.WFR:
        out["wfr"] = J.get_result(GPU, G.WFR, nd * N, np.complex64).reshape(shp)
    for flag, key, dt in ((G.IMG_AVG, "img_avg", np.float32), (G.DIF_AVG, "dif_avg", np.float32),
                          (G.WFR_AVG, "wfr_avg", np.complex64), (G.WFF_AVG, "wff_avg", np.complex64)):
        if im & flag:
            arr, w = J.get_avg_result(GPU, flag, nd * N, dt)
            out[key] = arr.reshape(shp)
            out[key + "_w"] = w
    if im & (G.WFR_AVG | G.WFF_AVG):   # ReadoutDetAvg of the averaged waves
        for flag, key, cnt in ((G.INT, "rda_int", nd * c["ndet"]), (G.IMG, "rda_img", nd * N),
                               (G.DIF, "rda_dif", nd * N)):
            if im & flag:
                e, arr, w = J.readout_det_avg(flag, cnt)
                assert e == 0, e
                out[key] = arr
                out["rda_w"] = w
    return c, out


def synthetic_specimen(nx, ny, nslc_types, nvar, seed, max_phase=1.5):
    """Seeded smooth random-phase gratings t = exp(i phi) (phi smoothed noise)."""
    rng = np.random.default_rng(seed)
    pgr = []
    ky = np.fft.fftfreq(ny)[:, None]
    kx = np.fft.fftfreq(nx)[None, :]
    filt = np.exp(-(kx ** 2 + ky ** 2) / (2 * 0.05 ** 2))
    for _ in range(nslc_types):
        g = []
        for _ in range(nvar):
            ph = np.fft.ifft2(np.fft.fft2(rng.normal(size=(ny, nx))) * filt).real
            ph = (ph - ph.min()) / (ph.max() - ph.min() + 1e-30) * max_phase
            g.append(np.exp(1j * np.mod(ph, 2 * np.pi)))
        pgr.append(np.asarray(g).astype(np.complex64))
    return pgr
