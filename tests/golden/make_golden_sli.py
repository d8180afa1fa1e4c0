"""Generate tests/golden/ref_slice_16x12.sli: an EMS slice file whose header
is written by the reference bench driver's prm_slice_file_info::save_ems_header
(test/JMSBench1/prm_slice_file_info.cpp) through oracle/_ref, with two seeded
16 x 12 grating variants.  It pins the product's slice-file reader.

Usage:  python tests/golden/make_golden_sli.py      (needs the reference sources)
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import ref  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_slice_16x12.sli")
PARAMS = dict(thickness=0.19525, ekv=300.0, sx=0.781, sy=0.5858, title="SrTiO3 [001] z=0 test", content=0)


def gratings():
    rng = np.random.default_rng(20261206)
    return np.exp(1j * rng.uniform(0, 1, (2, 12, 16))).astype(np.complex64)


def main():
    if not ref.available():
        ref.build()
    ref.sli_write(OUT, gratings(), **PARAMS)
    print(OUT, os.path.getsize(OUT))


if __name__ == "__main__":
    main()
