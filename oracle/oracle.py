"""ctypes front end of the FP64 multislice oracle (oracle/jms_oracle.cpp).

TEST INFRASTRUCTURE ONLY.  tests/, ``__graft_entry__.smoke()`` and bench.py's
CPU-baseline / error legs call it as the checker; the product never imports
it.  Every function names the reference routine it restates (file:line in the
reference project).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libjms_oracle.so")

_i = C.c_int
_d = C.c_double
_p = C.c_void_p
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)
_dp = C.POINTER(C.c_double)

_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.or_fft2d.argtypes = [_dp, _i, _i, _i]
        L.or_fft2d.restype = None
        L.or_detection_planes.argtypes = [_i, _i, _ip]
        L.or_detection_planes.restype = _i
        L.or_rng_create.argtypes = [_i]
        L.or_rng_create.restype = _p
        L.or_rng_destroy.argtypes = [_p]
        L.or_rng_destroy.restype = None
        L.or_variant_sequence.argtypes = [_p, _i, _ip, _i, _ip, _ip]
        L.or_variant_sequence.restype = _i
        L.or_offset.argtypes = [_i, _i, _d, _d, _d, _fp, _d, _d, _d, _fp, _i, _i, _dp]
        L.or_offset.restype = None
        L.or_multislice.argtypes = [_i, _i, _dp, _i, _i, _fp, _i, _i, _ip, _fp, _ip, _ip,
                                    _i, _fp, _ip, _ip, _i, _d, _dp, _dp, _dp, _dp, _dp, _ip]
        _f = C.c_float
        L.or_plasmon_shifts.argtypes = [_p, _i, _i, _fp, _f, _f, _f, _f, _f, C.c_uint, _ip]
        L.or_plasmon_shifts.restype = _i
        L.or_multislice.restype = _i
        L.or_pgr.argtypes = [_i, _i, _d, _d, _d, _i, _dp, _fp, _ip, _i, _i, _d, _fp, _i, _i, _dp]
        L.or_pgr.restype = _i
        _lib = L
    return _lib


def _f32(a):
    a = np.ascontiguousarray(a)
    if a.dtype == np.complex64:
        return a, a.ctypes.data_as(_fp)
    a = np.ascontiguousarray(a, np.float32)
    return a, a.ctypes.data_as(_fp)


def _i32(a):
    a = np.ascontiguousarray(a, np.int32)
    return a, a.ctypes.data_as(_ip)


def fft2d(z: np.ndarray, sign: int) -> np.ndarray:
    """Unnormalised 2-D C2C transform in FP64 (MKL DFTI convention,
    src/JFFTMKLcore.cpp:176,213): sign -1 forward, +1 backward."""
    w = np.ascontiguousarray(z, np.complex128).copy()
    ny, nx = w.shape
    lib().or_fft2d(w.ctypes.data_as(_dp), nx, ny, sign)
    return w


def detection_planes(ndetper: int, nobjslc: int):
    """SetDetectionPlanes (src/JMultiSlice.cpp:579-626)."""
    out = np.zeros(nobjslc + 1, np.int32)
    n = lib().or_detection_planes(ndetper, nobjslc, out.ctypes.data_as(_ip))
    return n, out


class Rng:
    """CRng restated (src/rng.cpp:30-74)."""

    def __init__(self, seed: int):
        self.h = lib().or_rng_create(seed)

    def __del__(self):
        try:
            lib().or_rng_destroy(self.h)
        except Exception:
            pass

    def plasmon_shifts(self, dt, ax, ay, q_e, q_c, mfp, nexmax, islc0=0) -> np.ndarray:
        """One plasmon Monte-Carlo path (CJPlasmonMC::ScatGridMC per slice) from
        this generator: [nobjslc, 2] pixel shifts."""
        d, pd = _f32(dt)
        out = np.zeros((len(d), 2), np.int32)
        e = lib().or_plasmon_shifts(self.h, len(d), islc0, pd, ax, ay, q_e, q_c, mfp, nexmax, out.ctypes.data_as(_ip))
        assert e == 0
        return out

    def variant_sequence(self, nvarslc, objslc) -> np.ndarray:
        """GetRandomVariantSequence (src/JMultiSlice.cpp:1571-1676)."""
        nv, pnv = _i32(nvarslc)
        ob, pob = _i32(objslc)
        out = np.zeros(len(ob), np.int32)
        e = lib().or_variant_sequence(self.h, len(nv), pnv, len(ob), pob, out.ctypes.data_as(_ip))
        assert e == 0
        return out


def offset(wav0, a, b, wl, dx, dy, dz=0.0, cppl=None, ibtx=0, ibty=0) -> np.ndarray:
    """OffsetIncomingWave, CPU branch (src/JMultiSlice.cpp:1999-2031), FP64."""
    w0, pw0 = _f32(np.asarray(wav0, np.complex64))
    ny, nx = w0.shape
    cp, pcp = (None, None) if cppl is None else _f32(cppl)
    out = np.zeros((ny, nx), np.complex128)
    lib().or_offset(nx, ny, a, b, wl, pw0, dx, dy, dz, pcp, ibtx, ibty, out.ctypes.data_as(_dp))
    return out


def multislice(wav, pgr_pool, pgr_idx, pro_pool, pro_idx, det_objslc, ndetslc, det=None, masks=None,
               imagedet=1, weight=1.0, islc0=0, acc=None, shifts=None):
    """One CPUMultislice run (src/JMultiSlice.cpp:3589-3720) in FP64.

    wav: complex Fourier-space entrance wave [ny, nx] (offset applied).
    pgr_pool [k, npgy, npgx] complex64 with pgr_idx[jslc] selecting the grating
    of object slice jslc; pro_pool [m, ny, nx] with pro_idx likewise.
    det: float [ndet, ny, nx]; masks: list of int arrays (empty = no mask).
    acc: dict of accumulators to add into (accmode 1), else fresh zeros.
    shifts: [nobjslc, 2] plasmon pixel shifts of the spectrum per slice, or None.
    Returns dict with det_int [ndetslc, ndet], dif, img, wff, wfr.
    """
    w = np.ascontiguousarray(wav, np.complex128).copy()
    ny, nx = w.shape
    N = nx * ny
    nobjslc = len(pgr_idx)
    pg, ppg = _f32(np.asarray(pgr_pool, np.complex64))
    npgy, npgx = pg.shape[-2], pg.shape[-1]
    pr, ppr = _f32(np.asarray(pro_pool, np.complex64))
    gi, pgi = _i32(pgr_idx)
    ri, pri = _i32(pro_idx)
    dh, pdh = _i32(det_objslc)
    ndet = 0 if det is None else int(np.asarray(det).shape[0])
    dt, pdt = _f32(np.zeros((1, ny, nx), np.float32) if det is None else det)
    if masks is None:
        masks = [np.zeros(0, np.int32)] * max(ndet, 1)
    ml, pml = _i32([len(m) for m in masks])
    mk, pmk = _i32(np.concatenate([np.asarray(m, np.int32) for m in masks] + [np.zeros(1, np.int32)]))
    if acc is None:
        acc = {
            "det_int": np.zeros((ndetslc, max(ndet, 1)), np.float64),
            "dif": np.zeros((ndetslc, ny, nx), np.float64),
            "img": np.zeros((ndetslc, ny, nx), np.float64),
            "wff": np.zeros((ndetslc, ny, nx), np.complex128),
            "wfr": np.zeros((ndetslc, ny, nx), np.complex128),
        }
    sh, psh = (None, None) if shifts is None else _i32(np.asarray(shifts).reshape(-1))
    e = lib().or_multislice(nx, ny, w.ctypes.data_as(_dp), nobjslc, islc0, ppg, npgx, npgy, pgi, ppr, pri, pdh,
                            ndet, pdt, pml, pmk, imagedet, weight,
                            acc["det_int"].ctypes.data_as(_dp), acc["dif"].ctypes.data_as(_dp),
                            acc["img"].ctypes.data_as(_dp), acc["wff"].ctypes.data_as(_dp),
                            acc["wfr"].ctypes.data_as(_dp), psh)
    assert e == 0
    acc["wave"] = w
    return acc


def pgr(nx, ny, a, b, wl, pos, occ, atype, ff, sk, bwl_pot=0, bwl_pgr=1) -> np.ndarray:
    """Phase grating of CJEElaSca::CalculatePhasegratingCPU (src/JEElaSca.cpp:812-976)
    in FP64.  pos [natom, 2] fractional (x/a, y/b) of the atoms as placed;
    occ, atype per atom; ff complex [ntype, nk] radial form factors sampled
    every sk 1/nm.  Returns complex128 [ny, nx]."""
    natom = len(occ)
    p = np.ascontiguousarray(pos, np.float64).reshape(natom, 2)
    o, po = _f32(occ)
    t, pt = _i32(atype)
    f, pf = _f32(np.asarray(ff, np.complex64))
    ntype, nk = f.shape
    out = np.zeros((ny, nx), np.complex128)
    e = lib().or_pgr(nx, ny, a, b, wl, natom, p.ctypes.data_as(_dp), po, pt, ntype, nk, sk, pf, bwl_pot, bwl_pgr,
                     out.ctypes.data_as(_dp))
    assert e == 0, e
    return out
