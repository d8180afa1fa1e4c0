"""Generate tests/golden/ref_golden.npz from the reference compiled here.

Runs the reference JMultiSliceLib (oracle/_ref/libjms_ref.so, built by
``make -C oracle ref`` from the reference sources) on small seeded cases and
stores its outputs: electron wavelengths, probe / propagator / ring-detector
generators, detection-plane hashes, the Fourier unscramble hash, frozen-phonon
variant draws and complete CPUMultislice runs (integrated detectors,
diffraction, image and wave readouts, averaging channels).  The reference has
no tests or golden data of its own, so these vectors are the parity pins for
both the FP64 oracle and the CUDA product.

Usage:  python tests/golden/make_golden.py      (needs the reference sources)
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import ref  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_golden.npz")
CPU = ref.CODE_CPU

# detection flags (src/JMultiSlice.h:139-149)
INT, IMG, DIF, WFR, WFF = 1, 2, 4, 8, 16
IMG_AVG, DIF_AVG, WFR_AVG, WFF_AVG = 32, 64, 128, 256

PROBE_CASES = {
    # name: (alpha mrad, alpha_rs, x0, y0, asym, adir deg, btx, bty, {abrr index: (x, y)} [nm])
    "p0": (25.0, 0.03, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, {}),
    "p1": (22.0, 0.03, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, {5: (1000.0, 0.0)}),
    "p2": (20.0, 0.05, 1.0, -0.5, 0.1, 30.0, 2.0, 1.0,
           {1: (5.0, 0.0), 2: (3.0, -2.0), 3: (50.0, 30.0), 4: (20.0, 10.0), 5: (1.0e3, 0.0),
            7: (2.0e3, -1.0e3), 11: (1.0e5, 0.0), 19: (3.0e7, 0.0)}),
}


def abrr_array(d):
    a = np.zeros(48, np.float32)
    for k, (x, y) in d.items():
        a[2 * k] = x
        a[2 * k + 1] = y
    return a


def generators(g):
    R = ref.RefJMS()
    for kv in (80.0, 200.0, 300.0):
        g[f"wl_{int(kv)}"] = np.float32(R.set_high_tension(kv))
    R.set_high_tension(300.0)
    nx, ny, a, b = 64, 48, 1.5, 1.2
    R.set_grid(nx, ny, a, b, 0.39)
    for name, (al, rs, x0, y0, asy, adir, btx, bty, ab) in PROBE_CASES.items():
        g[f"probe_{name}"] = R.calc_probe(al, rs, x0, y0, asy, adir, btx, bty, abrr_array(ab))
    DETS = [(0, 10, 0, 0, 0, 0, 0), (20, 50, 0, 0, 0, 0, 0), (80, 200, 0, 0, 0, 0, 0),
            (30, 60, 45, 135, 0, 0, 0), (10, 40, -30, 300, 0, 0, 0), (0, 25, 0, 0, 5, -3, 0),
            (20, 60, 0, 0, 0, 0, 1), (20, 60, 0, 0, 0, 0, 2)]
    for nt in (0, 1):
        g[f"pro_t{nt}"] = R.calc_propagator(0.19525, 0.0, 0.0, nt)
        g[f"pro_t{nt}_tilt"] = R.calc_propagator(0.25, 0.5, -0.3, nt)
        # ring detectors depend on the type of the last propagator computed
        for i, (b0, b1, f0, f1, tx, ty, km) in enumerate(DETS):
            det, msk = R.calc_ring_detector(b0, b1, f0, f1, tx, ty, km)
            g[f"det_t{nt}_{i}"] = det
            g[f"msk_t{nt}_{i}"] = msk
    g["det_params"] = np.array(DETS, np.float32)
    plist = [(0, 10), (5, 12), (10, 100), (20, 200), (3, 3), (7, 1), (4, 0), (0, 0)]
    for ndetper, nobj in plist:
        n, h = R.detection_planes(ndetper, nobj)
        g[f"planes_{ndetper}_{nobj}"] = h
        g[f"nplanes_{ndetper}_{nobj}"] = np.int32(n)
    g["planes_list"] = np.array(plist, np.int32)
    R.close()


def variant_draws(g):
    nvar = np.array([3, 1, 4, 2], np.int32)
    rng = np.random.default_rng(20261203)
    objslc = rng.integers(0, 4, 40).astype(np.int32)
    g["var_nvar"] = nvar
    g["var_objslc"] = objslc
    for seed in (11, 12):
        R = ref.RefJMS()
        R.set_high_tension(300.0)
        R.set_grid(8, 8, 1.0, 1.0, 1.0)
        R.setup(CPU, nvar, objslc, [0, 0, 0, 0], 0, 0, INT)
        R.seed(seed)
        g[f"var_seed{seed}"] = np.stack([R.variant_sequence(len(objslc)) for _ in range(3)])
        R.close()


def make_case(g, name, nx, ny, a, b, kv, nvar, objslc, thick, proidx, protype, tilt, dets, ndetper,
              imagedet, runs, seed, npg=None, probe=(25.0, {}), islc0=0, cppl_seed=None, avg_reads=(),
              plasmon=None, slcthick=None):
    """Set up one reference object (CPU code), run `runs` = [(dx,dy,dz,ibtx,ibty,accmode,weight)]."""
    rng = np.random.default_rng(seed)
    R = ref.RefJMS()
    wl = R.set_high_tension(kv)
    R.set_grid(nx, ny, a, b, 0.4)
    pros = [R.calc_propagator(t, tilt[0], tilt[1], protype) for t in thick]
    detarr, masks = [], []
    for (b0, b1, f0, f1, tx, ty, km, use_mask) in dets:
        d, m = R.calc_ring_detector(b0, b1, f0, f1, tx, ty, km)
        detarr.append(d)
        masks.append(m if use_mask else np.zeros(0, np.int32))
    wav0 = R.calc_probe(probe[0], abrr=abrr_array(probe[1]))
    npgx, npgy = (nx, ny) if npg is None else npg
    R.setup(CPU, nvar, objslc, proidx, ndetper, len(dets), imagedet, 1, npg=(npgx, npgy))
    grs = []
    for s, nv in enumerate(nvar):
        ph = rng.uniform(0.0, 1.2, (nv, npgy, npgx))
        gr = (np.exp(1j * ph) * rng.uniform(0.97, 1.0, (nv, npgy, npgx))).astype(np.complex64)
        grs.append(gr)
        R.set_phase_grating(CPU, s, gr)
    for i, p in enumerate(pros):
        R.set_propagator(CPU, i, p)
    for i, (d, m) in enumerate(zip(detarr, masks)):
        R.set_detector(CPU, i, d, m)
    R.init_core(CPU, 1)
    R.set_incident_wave(CPU, wav0)
    cppl = None
    if cppl_seed is not None:
        cppl = np.random.default_rng(cppl_seed).uniform(-0.5, 0.5, (ny, nx)).astype(np.float32)
        R.set_phaseplate(CPU, cppl)
    if slcthick is not None:
        for s_, t_ in enumerate(slcthick):
            R.set_slice_thickness(s_, t_)
    if plasmon is not None:
        R.set_plasmon(1, *plasmon)
    R.seed(seed)
    for (dx, dy, dz, ibtx, ibty, accmode, w) in runs:
        assert R.offset(CPU, dx, dy, dz, 0, ibtx, ibty) == 0
        e = R.cpu_multislice(islc0, accmode, w, 0)
        assert e == 0, e
    nd = R.num_det_planes()
    N = nx * ny
    p = f"{name}_"
    g[p + "cfg"] = np.array([nx, ny, npgx, npgy, protype, ndetper, imagedet, seed, islc0, len(dets)], np.int32)
    g[p + "cell"] = np.array([a, b, kv, wl, tilt[0], tilt[1]], np.float32)
    g[p + "nvar"] = np.array(nvar, np.int32)
    g[p + "objslc"] = np.array(objslc, np.int32)
    g[p + "thick"] = np.array(thick, np.float32)
    g[p + "proidx"] = np.array(proidx, np.int32)
    g[p + "dets"] = np.array(dets, np.float32)
    g[p + "runs"] = np.array(runs, np.float32)
    g[p + "probe"] = wav0
    for s, gr in enumerate(grs):
        g[p + f"pgr{s}"] = gr
    for i, pr in enumerate(pros):
        g[p + f"pro{i}"] = pr
    for i, (d, m) in enumerate(zip(detarr, masks)):
        g[p + f"det{i}"] = d
        g[p + f"msk{i}"] = m
    if cppl is not None:
        g[p + "cppl"] = cppl
    if plasmon is not None:
        g[p + "plasmon"] = np.array(plasmon, np.float32)
        g[p + "slcthick"] = np.array(slcthick, np.float32)
    g[p + "ndetslc"] = np.int32(nd)
    if imagedet & INT:
        g[p + "det_int"] = R.get_result(CPU, INT, nd * len(dets)).reshape(nd, len(dets))
    if imagedet & DIF:
        g[p + "dif"] = R.get_result(CPU, DIF, nd * N).reshape(nd, ny, nx)
    if imagedet & IMG:
        g[p + "img"] = R.get_result(CPU, IMG, nd * N).reshape(nd, ny, nx)
    if imagedet & WFF:
        g[p + "wff"] = R.get_result(CPU, WFF, nd * N, dtype=np.complex64).reshape(nd, ny, nx)
    if imagedet & WFR:
        g[p + "wfr"] = R.get_result(CPU, WFR, nd * N, dtype=np.complex64).reshape(nd, ny, nx)
    for flag, key, dt in ((IMG_AVG, "img_avg", np.float32), (DIF_AVG, "dif_avg", np.float32),
                          (WFR_AVG, "wfr_avg", np.complex64), (WFF_AVG, "wff_avg", np.complex64)):
        if imagedet & flag:
            arr, wgt = R.get_avg_result(CPU, flag, nd * N, dtype=dt)
            g[p + key] = arr.reshape(nd, ny, nx)
            g[p + key + "_w"] = np.float32(wgt)
    if name == "msa":
        g[p + "unscramble"] = R.unscramble_hash()
    if imagedet & (WFR_AVG | WFF_AVG):   # CJMultiSlice::ReadoutDetAvg of the averaged waves
        for flag, key, cnt in ((INT, "rda_int", nd * len(dets)), (IMG, "rda_img", nd * N), (DIF, "rda_dif", nd * N)):
            if imagedet & flag:
                e, arr, wgt = R.readout_det_avg(CPU, flag, cnt)
                assert e == 0, e
                g[p + key] = arr
                g[p + "rda_w"] = np.float32(wgt)
    R.close()


def multislice_cases(g):
    ring = [(0, 10, 0, 0, 0, 0, 0, 1), (20, 50, 0, 0, 0, 0, 0, 1), (80, 200, 0, 0, 0, 0, 0, 0),
            (20, 60, 0, 0, 0, 0, 1, 1)]
    # A: square grid, Fresnel propagators of two thicknesses, masked / unmasked
    # and signed (k-moment) detectors, all plain readouts, two accumulating runs.
    make_case(g, "msa", 64, 64, 1.1715, 1.1715, 300.0, [3, 2, 1], [i % 3 for i in range(12)],
              [0.19525, 0.3], [0, 0, 1], 1, (0.0, 0.0), ring, 5, INT | IMG | DIF | WFR | WFF,
              [(0.3, 0.2, 0.0, 0, 0, 0, 0.5), (0.1, 0.4, 1.0, 0, 0, 1, 0.5)], 5, probe=(22.0, {5: (1000.0, 0.0)}))
    # B: non-square grid, planar propagator with object tilt, exit-plane only,
    # segment and off-centre detectors.
    segs = [(0, 25, 0, 0, 0, 0, 0, 1), (30, 80, 45, 135, 0, 0, 0, 1), (10, 60, 0, 0, 4, -2, 0, 1)]
    make_case(g, "msb", 48, 40, 1.0, 0.85, 200.0, [2, 2], [0, 1, 0, 1, 1, 0, 1], [0.2], [0, 0], 0, (0.4, -0.2),
              segs, 0, INT | DIF | WFF, [(0.21, 0.13, 2.0, 0, 0, 0, 1.0)], 9, probe=(20.0, {2: (2.0, 1.0)}))
    # C: sub-frame gratings (32x16 repeated over a 64x32 grid).
    make_case(g, "msc", 64, 32, 1.6, 0.8, 300.0, [2, 1], [0, 1, 0, 1, 0, 1], [0.2], [0, 0], 1, (0.0, 0.0),
              ring[:3], 2, INT | DIF, [(0.05, 0.1, 0.0, 0, 0, 0, 1.0)], 13, npg=(32, 16))
    # D: averaging channels over three runs of accmode 0.
    make_case(g, "msd", 32, 32, 0.9, 0.9, 300.0, [3], [0] * 8, [0.2], [0], 1, (0.0, 0.0), ring[:2], 4,
              INT | IMG_AVG | DIF_AVG | WFR_AVG | WFF_AVG,
              [(0.1, 0.1, 0.0, 0, 0, 0, 1 / 3), (0.2, 0.3, 0.0, 0, 0, 0, 1 / 3), (0.4, 0.0, 0.0, 0, 0, 0, 1 / 3)], 17)
    # G: readouts of the averaged waves (ReadoutDetAvg) over three weighted runs.
    make_case(g, "msg", 48, 48, 1.0, 1.0, 300.0, [3, 2], [0, 1] * 5, [0.19525], [0, 0], 1, (0.0, 0.0), ring[:3],
              5, INT | IMG | DIF | WFR_AVG | WFF_AVG,
              [(0.1, 0.2, 0.0, 0, 0, 0, 0.5), (0.3, 0.1, 0.0, 0, 0, 1, 0.25), (0.2, 0.4, 0.0, 0, 0, 1, 0.25)], 29)
    # H: bulk plasmon Monte-Carlo (short mean free path so that several
    # excitations happen): q_e, q_c [1/nm], mfp [nm], at most 3 excitations;
    # four accumulating runs, each its own Monte-Carlo path.
    make_case(g, "msh", 64, 64, 1.5, 1.5, 300.0, [2, 2], [0, 1] * 8, [0.2], [0, 0], 1, (0.0, 0.0), ring[:3],
              4, INT | DIF | WFF, [(0.3, 0.4, 0.0, 0, 0, 0, 0.25), (0.3, 0.4, 0.0, 0, 0, 1, 0.25),
                                  (0.3, 0.4, 0.0, 0, 0, 1, 0.25), (0.3, 0.4, 0.0, 0, 0, 1, 0.25)], 31,
              plasmon=(0.8, 6.0, 0.6, 3), slcthick=[0.2, 0.2])
    # E: start slice > 0, probe beam tilt in pixels and a constant phase plate.
    make_case(g, "mse", 64, 64, 1.2, 1.2, 300.0, [2, 2], [0, 1] * 5, [0.19525], [0, 0], 1, (0.0, 0.0), ring[:3],
              3, INT | DIF | IMG, [(0.2, 0.1, 0.5, 2, -1, 0, 1.0)], 21, islc0=4, cppl_seed=3)
    # F: a longer run on 128x128 for FP32 accumulation over 40 slices.
    make_case(g, "msf", 128, 128, 2.343, 2.343, 300.0, [2, 2, 2, 2], [i % 4 for i in range(40)], [0.19525],
              [0, 0, 0, 0], 1, (0.0, 0.0), ring[:3], 10, INT | DIF, [(1.1, 0.9, 0.0, 0, 0, 0, 1.0)], 23,
              probe=(22.0, {5: (1000.0, 0.0)}))


def main():
    if not ref.build():
        print("reference library not available")
        return 1
    g: dict = {}
    generators(g)
    variant_draws(g)
    multislice_cases(g)
    np.savez_compressed(OUT, **g)
    print(f"wrote {OUT}: {len(g)} arrays, {os.path.getsize(OUT) / 1e6:.2f} MB")
    return 0


if __name__ == "__main__":
    sys.exit(main())
