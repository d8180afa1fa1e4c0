"""Generate tests/golden/ref_pgr.npz: phase gratings of the reference's CJEElaSca.

Runs the reference's phase-grating calculation (CJEElaSca on its CPU path,
src/JEElaSca.cpp:812-976, with Weickenmeier-Kohl form factors from
src/wekoscat.cpp) through oracle/_ref/libjms_ref.so on small perovskite
slices and stores inputs, the prepared radial form-factor tables and the
gratings.  These pin the FP64 oracle's restatement (tests/test_pgr_oracle.py)
and the on-device generator (tests/test_pgr_gpu.py).

Usage:  python tests/golden/make_golden_pgr.py      (needs the reference sources)
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import ref  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_pgr.npz")
A0 = 0.3905   # nm


def layer(ncx, ncy, sites):
    """sites: (Z, fx, fy, biso nm^2, occ) per unit cell -> per-atom arrays."""
    Z, bi, oc, pos = [], [], [], []
    for i in range(ncx):
        for j in range(ncy):
            for (z, fx, fy, b, o) in sites:
                Z.append(z)
                bi.append(b)
                oc.append(o)
                pos.append(((i + fx) / ncx, (j + fy) / ncy, 0.0))
    return np.array(Z, np.int32), np.array(bi, np.float32), np.array(oc, np.float32), np.array(pos, np.float32)


CASES = {
    # name: (nx, ny, ncx, ncy, sites, thermal, absorb, abf)
    "g0": (64, 64, 3, 3, [(38, 0.0, 0.0, 0.0055, 1.0), (8, 0.5, 0.5, 0.0070, 1.0)], 0, 0, 0.0),
    "g1": (96, 64, 3, 2, [(22, 0.5, 0.5, 0.0040, 1.0), (8, 0.5, 0.0, 0.0070, 1.0), (8, 0.0, 0.5, 0.0070, 1.0)],
           1, 1, 0.1),
    "g2": (64, 64, 2, 2, [(57, 0.0, 0.0, 0.0050, 0.5), (38, 0.0, 0.0, 0.0060, 0.5), (8, 0.5, 0.5, 0.0070, 1.0)],
           1, 2, 0.0),
}


def main():
    if not ref.available():
        ref.build()
    g = {}
    R = ref.RefJMS()
    wl = R.set_high_tension(300.0)
    R.close()
    for name, (nx, ny, ncx, ncy, sites, thermal, absorb, abf) in CASES.items():
        Z, bi, oc, pos = layer(ncx, ncy, sites)
        a, b, c = ncx * A0, ncy * A0, A0 / 2
        pgr, at, ff, sk, _ = ref.pgr(nx, ny, a, b, c, 300.0, Z, bi, oc, pos, thermal=thermal, absorb=absorb,
                                    abf=abf)
        for k, v in dict(nx=nx, ny=ny, a=a, b=b, c=c, thermal=thermal, absorb=absorb, abf=abf, Z=Z, biso=bi, occ=oc,
                         pos=pos, atype=at, ff=ff, sk=sk, pgr=pgr[0], wl=wl).items():
            g[f"{name}_{k}"] = np.asarray(v)
    np.savez_compressed(OUT, **g)
    print(OUT, os.path.getsize(OUT))


if __name__ == "__main__":
    main()
