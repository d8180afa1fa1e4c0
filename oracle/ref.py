"""ctypes loader for the compiled reference (oracle/_ref/libjms_ref.so).

TEST INFRASTRUCTURE ONLY: used by tests/golden/make_golden.py to produce golden
vectors, by tests to pin the FP64 oracle, and by bench.py's reference arm to
time the reference CPU path (CJMultiSlice::CPUMultislice, src/JMultiSlice.cpp:
3589-3720, on MKL DFTI).  The product never imports this module.

The library is built by ``make -C oracle ref`` from the reference sources
(see oracle/Makefile); on a machine without those sources only a prebuilt
``oracle/_ref/libjms_ref.so`` can be used.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libjms_ref.so")

CODE_CPU = 1
CODE_GPU = 2

_f = C.c_float
_i = C.c_int
_p = C.c_void_p
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)

_lib = None


def build(refroot: str | None = None) -> bool:
    """Build the reference library when the reference project is present
    (refroot, default: the JMS_REFERENCE environment variable)."""
    refroot = refroot or os.environ.get("JMS_REFERENCE", "")
    if not refroot or not os.path.isdir(os.path.join(refroot, "src")):
        return os.path.exists(LIB_PATH)
    subprocess.run(["make", "-s", "-C", HERE, "ref", f"JMS_REFERENCE={refroot}", "-j8"], check=True)
    return os.path.exists(LIB_PATH)


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"reference library missing: {LIB_PATH} (run make -C oracle ref)")
        # libtorch_cpu.so (which carries MKL) must be initialised by torch itself
        # before the reference library pulls it in; loading it behind numpy alone
        # aborts at interpreter exit.
        import torch  # noqa: F401
        L = C.CDLL(LIB_PATH)
        sig = {
            "ref_create": ([], _p),
            "ref_destroy": ([_p], None),
            "ref_set_high_tension": ([_p, _f], _f),
            "ref_set_grid": ([_p, _i, _i, _f, _f, _f], None),
            "ref_seed": ([_p, _i], None),
            "ref_phase_grating_setup": ([_p, _i, _i, _i, _i, _i, _ip], _i),
            "ref_object_slice_setup": ([_p, _i, _ip], _i),
            "ref_propagator_setup": ([_p, _i, _i, _ip], _i),
            "ref_detector_setup": ([_p, _i, _i, _i, _i, _i], _i),
            "ref_set_phase_grating": ([_p, _i, _i, _i, _fp], _i),
            "ref_set_propagator": ([_p, _i, _i, _fp], _i),
            "ref_set_detector": ([_p, _i, _i, _fp, _i, _ip], _i),
            "ref_init_core": ([_p, _i, _i], _i),
            "ref_set_incident_wave": ([_p, _i, _fp], _i),
            "ref_set_phaseplate": ([_p, _i, _fp], _i),
            "ref_offset_incoming_wave": ([_p, _i, _f, _f, _f, _i, _i, _i], _i),
            "ref_cpu_multislice": ([_p, _i, _i, _f, _i], _i),
            "ref_gpu_multislice": ([_p, _i, _i, _f], _i),
            "ref_get_result": ([_p, _i, _i, _fp, _i], _i),
            "ref_get_avg_result": ([_p, _i, _i, _fp, _fp, _i], _i),
            "ref_num_det_planes": ([_p], _i),
            "ref_unscramble_hash": ([_p, C.POINTER(C.c_uint)], _i),
            "ref_variant_sequence": ([_p, _ip], _i),
            "ref_cpu_wave": ([_p, _i, _fp, _i], None),
            "ref_detection_planes": ([_p, _i, _i, _ip], _i),
            "ref_cleanup": ([_p], _i),
            "ref_calc_probe": ([_p, _f, _f, _f, _f, _f, _f, _f, _f, _fp, _i, _fp], _i),
            "ref_calc_propagator": ([_p, _f, _f, _f, _i, _fp], _i),
            "ref_calc_ring_detector": ([_p, _f, _f, _f, _f, _f, _f, C.c_char_p, _fp, _ip, _ip, _i], _i),
            "ref_cpu_scan": ([C.POINTER(_p), _i, _i, _fp, _i, _i, _fp], _i),
            "ref_gpu_scan": ([_p, _i, _fp, _i, _i, _fp, C.POINTER(C.c_double)], _i),
            "ref_set_slice_thickness": ([_p, _i, _f], None),
            "ref_set_plasmon": ([_p, _i, _f, _f, _f, C.c_uint], None),
            "ref_sli_read_header": ([C.c_char_p, _ip, C.POINTER(C.c_ulonglong), _fp, C.c_char_p], _i),
            "ref_sli_write": ([C.c_char_p, _i, _i, _i, _i, _f, _f, _f, _f, C.c_char_p, _fp], _i),
            "ref_readout_det_avg": ([_p, _i, _i, _fp, _fp, _i], _i),
            "ref_pgr": ([_i, _i, _f, _f, _f, _f, _i, _i, _f, _i, _ip, _fp, _fp, _fp, _i, _i, _fp, _ip, _fp, _ip, _fp,
                         _ip, C.POINTER(C.c_double)], _i),
        }
        for name, (args, res) in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def fptr(a: np.ndarray):
    assert a.dtype in (np.float32, np.complex64) and a.flags.c_contiguous
    return a.ctypes.data_as(_fp)


def iptr(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_ip)


class RefJMS:
    """One reference CJMultiSlice object (src/JMultiSlice.h:185)."""

    def __init__(self):
        self.L = lib()
        self.h = self.L.ref_create()

    def close(self):
        if self.h:
            self.L.ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # physics / grid
    def set_high_tension(self, ht):
        return self.L.ref_set_high_tension(self.h, ht)

    def set_grid(self, nx, ny, a, b, c):
        self.L.ref_set_grid(self.h, nx, ny, a, b, c)
        self.nx, self.ny = nx, ny

    def seed(self, s):
        self.L.ref_seed(self.h, s)

    # generators
    def calc_probe(self, alpha, alpha_rs=0.03, x0=0.0, y0=0.0, asym=0.0, adir=0.0, btx=0.0, bty=0.0, abrr=None):
        ab = np.zeros(48, np.float32) if abrr is None else np.ascontiguousarray(abrr, np.float32)
        wav = np.zeros((self.ny, self.nx), np.complex64)
        e = self.L.ref_calc_probe(self.h, alpha, alpha_rs, x0, y0, asym, adir, btx, bty, fptr(ab), ab.size, fptr(wav))
        assert e == 0, e
        return wav

    def calc_propagator(self, fthick, otx=0.0, oty=0.0, ntype=0):
        pro = np.zeros((self.ny, self.nx), np.complex64)
        e = self.L.ref_calc_propagator(self.h, fthick, otx, oty, ntype, fptr(pro))
        assert e == 0, e
        return pro

    def calc_ring_detector(self, beta0, beta1, phi0=0.0, phi1=0.0, th0x=0.0, th0y=0.0, kmom1=0, profile=b""):
        det = np.zeros((self.ny, self.nx), np.float32)
        msk = np.zeros(self.nx * self.ny, np.int32)
        ml = C.c_int(0)
        e = self.L.ref_calc_ring_detector(self.h, beta0, beta1, phi0, phi1, th0x, th0y, profile,
                                          fptr(det), C.byref(ml), iptr(msk), kmom1)
        assert e == 0, e
        return det, msk[: ml.value].copy()

    # setup chain (JMultiSlice.h:77-97)
    def setup(self, code, nslcvar, objslc, proidx, ndetper, ndet, imagedet, nthreads=1, npg=None):
        nslcvar = np.ascontiguousarray(nslcvar, np.int32)
        objslc = np.ascontiguousarray(objslc, np.int32)
        proidx = np.ascontiguousarray(proidx, np.int32)
        npgx, npgy = (self.nx, self.ny) if npg is None else npg
        L, h = self.L, self.h
        assert L.ref_phase_grating_setup(h, code, npgx, npgy, len(nslcvar), int(nslcvar.max()), iptr(nslcvar)) == 0
        assert L.ref_object_slice_setup(h, len(objslc), iptr(objslc)) == 0
        assert L.ref_propagator_setup(h, code, int(proidx.max()) + 1, iptr(proidx)) == 0
        assert L.ref_detector_setup(h, code, ndetper, ndet, imagedet, nthreads) == 0
        self._keep = []

    def set_phase_grating(self, code, islc, pgr):
        pgr = np.ascontiguousarray(pgr, np.complex64)
        self._keep.append(pgr)  # the CPU path borrows the array
        nvar = pgr.shape[0] if pgr.ndim == 3 else 1
        assert self.L.ref_set_phase_grating(self.h, code, islc, nvar, fptr(pgr)) == 0

    def set_propagator(self, code, ipro, pro):
        pro = np.ascontiguousarray(pro, np.complex64)
        self._keep.append(pro)
        assert self.L.ref_set_propagator(self.h, code, ipro, fptr(pro)) == 0

    def set_detector(self, code, idet, det, msk=None):
        det = np.ascontiguousarray(det, np.float32)
        self._keep.append(det)
        if msk is None or len(msk) == 0:
            assert self.L.ref_set_detector(self.h, code, idet, fptr(det), 0, None) == 0
        else:
            msk = np.ascontiguousarray(msk, np.int32)
            self._keep.append(msk)
            assert self.L.ref_set_detector(self.h, code, idet, fptr(det), len(msk), iptr(msk)) == 0

    def init_core(self, code, nthreads=1):
        e = self.L.ref_init_core(self.h, code, nthreads)
        assert e == 0, e

    def set_incident_wave(self, code, wav):
        wav = np.ascontiguousarray(wav, np.complex64)
        assert self.L.ref_set_incident_wave(self.h, code, fptr(wav)) == 0

    def set_phaseplate(self, code, ppl):
        ppl = np.ascontiguousarray(ppl, np.float32)
        assert self.L.ref_set_phaseplate(self.h, code, fptr(ppl)) == 0

    def offset(self, code, dx, dy, dz=0.0, ithread=0, ibtx=0, ibty=0):
        return self.L.ref_offset_incoming_wave(self.h, code, dx, dy, dz, ithread, ibtx, ibty)

    def cpu_multislice(self, islc0=0, accmode=0, weight=1.0, ithread=0):
        return self.L.ref_cpu_multislice(self.h, islc0, accmode, weight, ithread)

    def gpu_multislice(self, islc0=0, accmode=0, weight=1.0):
        return self.L.ref_gpu_multislice(self.h, islc0, accmode, weight)

    def num_det_planes(self):
        return self.L.ref_num_det_planes(self.h)

    def get_result(self, code, which, count, ithread=0, dtype=np.float32):
        dst = np.zeros(count, dtype)
        self.L.ref_get_result(self.h, code, which, dst.view(np.float32).ctypes.data_as(_fp), ithread)
        return dst

    def get_avg_result(self, code, which, count, ithread=0, dtype=np.float32):
        dst = np.zeros(count, dtype)
        w = C.c_float(0)
        self.L.ref_get_avg_result(self.h, code, which, dst.view(np.float32).ctypes.data_as(_fp), C.byref(w), ithread)
        return dst, w.value

    def set_slice_thickness(self, islc, t):
        lib().ref_set_slice_thickness(self.h, islc, t)

    def set_plasmon(self, use, q_e, q_c, mfp, nexmax):
        lib().ref_set_plasmon(self.h, int(use), q_e, q_c, mfp, nexmax)

    def readout_det_avg(self, code, which, count, ithread=0):
        """CJMultiSlice::ReadoutDetAvg: (error, dst, weight)."""
        dst = np.zeros(count, np.float32)
        w = C.c_float(0)
        e = lib().ref_readout_det_avg(self.h, code, which, fptr(dst), C.byref(w), ithread)
        return e, dst, w.value

    def cpu_wave(self, ithread=0):
        out = np.zeros((self.ny, self.nx), np.complex64)
        self.L.ref_cpu_wave(self.h, ithread, fptr(out), self.nx * self.ny)
        return out

    def variant_sequence(self, nobjslc):
        out = np.zeros(nobjslc, np.int32)
        assert self.L.ref_variant_sequence(self.h, iptr(out)) == 0
        return out

    def unscramble_hash(self):
        out = np.zeros(self.nx * self.ny, np.uint32)
        self.L.ref_unscramble_hash(self.h, out.ctypes.data_as(C.POINTER(C.c_uint)))
        return out

    def detection_planes(self, ndetper, nobjslc):
        out = np.zeros(nobjslc + 1, np.int32)
        n = self.L.ref_detection_planes(self.h, ndetper, nobjslc, iptr(out))
        return n, out


def cpu_scan(objs, npos_xy: np.ndarray, nrepeat: int, ndetout: int) -> tuple[np.ndarray, int]:
    """Run the reference multi-threaded CPU scan; one RefJMS per thread."""
    import torch

    L = lib()
    arr = (C.c_void_p * len(objs))(*[o.h for o in objs])
    pos = np.ascontiguousarray(npos_xy, np.float32)
    out = np.zeros((pos.shape[0], ndetout), np.float32)
    # one MKL thread per transform (the reference links mkl_sequential); the
    # parallelism is one worker thread per CJMultiSlice object
    nt0 = torch.get_num_threads()
    torch.set_num_threads(1)
    try:
        e = L.ref_cpu_scan(arr, len(objs), pos.shape[0], fptr(pos), nrepeat, ndetout, fptr(out))
    finally:
        torch.set_num_threads(nt0)
    return out, e


def gpu_scan(obj, npos_xy: np.ndarray, nrepeat: int, ndetout: int) -> tuple[np.ndarray, float, int]:
    """The reference GPU path (GPUMultislice, cuFFT) over positions x nrepeat
    passes on one object set up for GPU code; returns (integrated detectors
    [npos, ndetout], seconds, error code)."""
    L = lib()
    pos = np.ascontiguousarray(npos_xy, np.float32)
    out = np.zeros((pos.shape[0], ndetout), np.float32)
    sec = C.c_double(0.0)
    e = L.ref_gpu_scan(obj.h, pos.shape[0], fptr(pos), nrepeat, ndetout, fptr(out), C.byref(sec))
    return out, sec.value, e


def pgr(nx, ny, a, b, c, ekv, Z, biso, occ, pos, thermal=0, absorb=0, abf=0.0, nrep=1, seed=0):
    """Phase grating(s) of one structure slice by the reference's CJEElaSca CPU
    path (src/JEElaSca.cpp:812-976): Z, biso [nm^2], occ per atom, pos [natom, 3]
    fractional.  Returns (pgr complex64 [nrep, ny, nx], atom_type [natom],
    ff complex64 [ntype, nk], sk, seconds)."""
    import torch  # noqa: F401  (MKL lives in libtorch_cpu)

    L = lib()
    natom = len(Z)
    Z = np.ascontiguousarray(Z, np.int32)
    biso = np.ascontiguousarray(biso, np.float32)
    occ = np.ascontiguousarray(occ, np.float32)
    pos = np.ascontiguousarray(pos, np.float32).reshape(natom, 3)
    out = np.zeros((nrep, ny, nx), np.complex64)
    at = np.zeros(natom, np.int32)
    cap = 12 * max(nx, ny)
    ff = np.zeros((natom, cap), np.complex64)
    nk = C.c_int(cap)
    sk = C.c_float(0)
    nt = C.c_int(0)
    sec = C.c_double(0)
    nt0 = torch.get_num_threads()
    torch.set_num_threads(1)
    try:
        e = L.ref_pgr(nx, ny, a, b, c, ekv, thermal, absorb, abf, natom, iptr(Z), fptr(biso), fptr(occ), fptr(pos),
                      nrep, seed, fptr(out), iptr(at), fptr(ff), C.byref(nk), C.byref(sk), C.byref(nt),
                      C.byref(sec))
    finally:
        torch.set_num_threads(nt0)
    assert e == 0, e
    return out, at, ff[:nt.value, :nk.value].copy(), sk.value, sec.value


def sli_read_header(path):
    """The bench driver's prm_slice_file_info::load_ems_header on a file."""
    ints = np.zeros(5, np.int32)
    offs = (C.c_ulonglong * 2)()
    f = np.zeros(4, np.float32)
    title = C.create_string_buffer(41)
    e = lib().ref_sli_read_header(os.fsencode(path), iptr(ints), offs, fptr(f), title)
    assert e == 0, e
    return {"nx": int(ints[0]), "ny": int(ints[1]), "nvar": int(ints[2]), "content": int(ints[3]),
            "version": int(ints[4]) & 0xFFFFFFFF, "data_offset": int(offs[0]), "table_offset": int(offs[1]),
            "thickness": float(f[0]), "ekv": float(f[1]), "sx": float(f[2]), "sy": float(f[3]),
            "title": title.value.decode("latin-1")}


def sli_write(path, pgr, thickness, ekv, sx, sy, title="", content=0):
    """A slice file whose header is written by prm_slice_file_info::save_ems_header."""
    g = np.ascontiguousarray(pgr, np.complex64)
    e = lib().ref_sli_write(os.fsencode(path), g.shape[2], g.shape[1], g.shape[0], content, thickness, ekv, sx, sy,
                            title.encode("latin-1"), fptr(g))
    assert e == 0, e
