"""Golden-vector helpers shared by the tests.

The fixtures in tests/golden/ref_golden.npz come from the reference compiled
here (tests/golden/make_golden.py).  ``oracle_case`` replays one golden
multislice case through the FP64 oracle: same gratings, propagators, detectors,
probe, offsets, weights and the same frozen-phonon variant draws (CRng with the
case's seed, src/rng.cpp:30-74).
"""
from __future__ import annotations

import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_golden.npz")
_cache = None

INT, IMG, DIF, WFR, WFF = 1, 2, 4, 8, 16
IMG_AVG, DIF_AVG, WFR_AVG, WFF_AVG = 32, 64, 128, 256
CASES = ("msa", "msb", "msc", "msd", "mse", "msf", "msg", "msh")


def golden():
    global _cache
    if _cache is None:
        with np.load(GOLDEN) as z:
            _cache = {k: z[k] for k in z.files}
    return _cache


def case(name: str) -> dict:
    g = golden()
    p = name + "_"
    c = {k[len(p):]: v for k, v in g.items() if k.startswith(p)}
    cfg = c["cfg"]
    c["nx"], c["ny"], c["npgx"], c["npgy"] = (int(v) for v in cfg[:4])
    c["protype"], c["ndetper"], c["imagedet"], c["seed"], c["islc0"], c["ndet"] = (int(v) for v in cfg[4:10])
    a, b, kv, wl, otx, oty = (float(v) for v in c["cell"])
    c.update(a=a, b=b, kv=kv, wl=wl)
    c["pgr"] = [c[f"pgr{s}"] for s in range(len(c["nvar"]))]
    c["pro"] = [c[f"pro{i}"] for i in range(int(c["proidx"].max()) + 1)]
    c["det"] = [c[f"det{i}"] for i in range(c["ndet"])]
    c["msk"] = [c[f"msk{i}"] for i in range(c["ndet"])]
    return c


def oracle_case(name: str) -> dict:
    from oracle import oracle as OR

    c = case(name)
    nobj = len(c["objslc"])
    ndetslc, hsh = OR.detection_planes(c["ndetper"], nobj)
    pool = np.concatenate(c["pgr"], 0)
    base = np.concatenate([[0], np.cumsum(c["nvar"])[:-1]]).astype(np.int64)
    rng = OR.Rng(c["seed"])
    acc = None
    avg = None
    det = np.stack(c["det"]) if c["ndet"] else None
    for (dx, dy, dz, ibtx, ibty, accmode, w) in c["runs"]:
        var = rng.variant_sequence(c["nvar"], c["objslc"])
        pidx = (base[c["objslc"]] + var).astype(np.int32)
        shifts = None
        if "plasmon" in c and c["islc0"] < nobj:   # one Monte-Carlo path per run, after the variant draw
            qe, qc, mfp, nmax = (float(v) for v in c["plasmon"])
            shifts = rng.plasmon_shifts(c["slcthick"][c["objslc"]], np.float32(c["a"]), np.float32(c["b"]), qe, qc,
                                        mfp, int(nmax), islc0=c["islc0"])
        wav = OR.offset(c["probe"], c["a"], c["b"], c["wl"], dx, dy, dz, c.get("cppl"), int(ibtx), int(ibty))
        if accmode == 0 or acc is None:
            acc = None
        res = OR.multislice(wav, pool, pidx, np.stack(c["pro"]), c["proidx"][c["objslc"]], hsh, ndetslc,
                            det=det, masks=c["msk"], imagedet=c["imagedet"], weight=float(w),
                            islc0=c["islc0"], acc=acc, shifts=shifts)
        acc = res
        # averaging channels are never cleared by accmode 0 (src/JMultiSlice.cpp:3128-3166)
        if c["imagedet"] & (IMG_AVG | DIF_AVG | WFR_AVG | WFF_AVG):
            if avg is None:
                avg = {k: np.zeros_like(v) for k, v in res.items() if k != "wave"}
                avg["w"] = 0.0
            one = OR.multislice(wav, pool, pidx, np.stack(c["pro"]), c["proidx"][c["objslc"]], hsh, ndetslc,
                                det=det, masks=c["msk"], imagedet=c["imagedet"], weight=float(w),
                                islc0=c["islc0"], shifts=shifts)
            for k in avg:
                if k != "w":
                    avg[k] += one[k]
            avg["w"] += float(w)
    acc["ndetslc"] = ndetslc
    acc["avg"] = avg
    return acc


def rel_err(a, b) -> float:
    a = np.asarray(a)
    b = np.asarray(b)
    den = np.abs(b).max()
    return float(np.abs(a - b).max() / (den if den > 0 else 1.0))
