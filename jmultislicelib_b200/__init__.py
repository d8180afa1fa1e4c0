"""jmultislicelib_b200 -- B200-native multislice hot path of JMultiSliceLib.

The product is the shared library ``libjms_b200.so`` (CUDA for sm_100a + C++
host code) with the C ABI of ``include/jms_b200.h``, a drop-in for the GPU
path of JMultiSliceLib's flat interface (src/JMultiSliceLib.h).  This module
is a thin ctypes binding of that ABI for Python callers (tests, bench); it
adds no computation of its own and raises if the library is not built --
there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libjms_b200.so")

CODE_CPU, CODE_GPU = 1, 2
INT, IMG, DIF, WFR, WFF = 1, 2, 4, 8, 16
IMG_AVG, DIF_AVG, WFR_AVG, WFF_AVG = 32, 64, 128, 256

_f, _i, _p = C.c_float, C.c_int, C.c_void_p
_fp, _ip, _dp = C.POINTER(C.c_float), C.POINTER(C.c_int), C.POINTER(C.c_double)


class JMSProbeParams(C.Structure):
    """CJProbeParams public data (src/JProbeGen.h:60-94), see include/jms_b200.h."""

    _fields_ = [("m_wl", _f), ("m_alpha", _f), ("m_alpha_rs", _f), ("m_alpha_x0", _f), ("m_alpha_y0", _f),
                ("m_alpha_asym", _f), ("m_alpha_adir", _f), ("m_btx", _f), ("m_bty", _f),
                ("m_source_width", _f), ("m_source_shape", _i), ("m_fspread_width", _f),
                ("m_fspread_kernel_width", _f), ("m_fspread_kernel_samples", _i), ("m_abrr_coeff", _fp)]


class JMSSliHeader(C.Structure):
    """EMS slice-file header fields (include/jms_b200.h)."""

    _fields_ = [("nx", _i), ("ny", _i), ("nvar", _i), ("content", _i), ("version", C.c_uint),
                ("data_offset", C.c_uint), ("table_offset", C.c_uint), ("thickness", _f), ("ekv", _f), ("sx", _f),
                ("sy", _f), ("swapped", _i), ("title", C.c_char * 41)]


# name -> (argtypes, restype) of every symbol declared in include/jms_b200.h
SIGNATURES = {
    "GetJMSVersion": ([], _f), "SetJMSDebugLevel": ([_i], _i), "SeedRngEx": ([_i], None),
    "SetHighTension": ([_f], _f), "GetHighTension": ([], _f), "GetWaveLength": ([], _f),
    "SetSupercellSize": ([_fp], None), "SetSupercellSizeABC": ([_f, _f, _f], None),
    "SetSliceThickness": ([_i, _f], None), "DiffractionDescan": ([_i], None),
    "SetPlasmonMC": ([_i, _f, _f, _f, C.c_uint], None),
    "SetDiffractionDescanN": ([_i, _i, _i, _i], None), "SetDiffractionDescan": ([_i, _f, _f, _i], None),
    "SetDiffractionDescanMRad": ([_i, _f, _f, _i], None),
    "SetGridSize": ([_i, _i], None), "GetGridSize": ([_ip, _ip], None),
    "GetDetetionSliceNum": ([], _i), "GetDetNum": ([], _i), "GetCPUNum": ([], _i), "GetGPUNum": ([], _i),
    "GetGPUName": ([_i, C.c_char_p], _i), "GetCurrentGPU": ([], _i), "SetCurrentGPU": ([_i], _i),
    "GetGPUStats": ([_i, _ip, _ip, _ip, C.POINTER(C.c_int64), C.POINTER(C.c_int64)], _i),
    "GetUnscrambleHash": ([C.POINTER(C.c_uint)], _i),
    "GetImageAveragingWeight": ([_i, _i], _f), "GetWaveAveragingWeight": ([_i, _i], _f),
    "PhaseGratingSetup": ([_i, _i, _i, _i, _i, _ip], _i), "ObjectSliceSetup": ([_i, _ip], _i),
    "PropagatorSetup": ([_i, _i, _ip], _i), "DetectorSetup": ([_i, _i, _i, _i, _i], _i),
    "InitCore": ([_i, _i], _i), "SetIncidentWave": ([_i, _fp], _i),
    "SetIncidentWavePhaseplate": ([_i, _fp, _i], _i), "ZeroIncidentWavePhaseplate": ([_i], _i),
    "SetSlicePhaseGratings": ([_i, _i, _i, _fp], _i), "SetPropagatorData": ([_i, _i, _fp], _i),
    "SetDetectorData": ([_i, _i, _fp, _i, _ip], _i), "SetGPUPgrLoading": ([_i], _i),
    "ResetImageAveraging": ([_i, _i], _i), "ResetWaveAveraging": ([_i, _i], _i),
    "CalculateProbeWaveFourier": ([C.POINTER(JMSProbeParams), _fp], _i),
    "SetIncomingWaveGPU": ([_fp, _i], _i), "SetIncomingWaveCPU": ([_fp, _i, _i], _i),
    "CalculatePropagator": ([_f, _f, _f, _fp, _i], _i),
    "CalculateRingDetector": ([_f, _f, _f, _f, _f, _f, C.c_char_p, _fp, _ip, _ip, _i], _i),
    "OffsetIncomingWave": ([_i, _f, _f, _f, _i, _i, _i], _i),
    "CPUMultislice": ([_i, _i, _f, _i], _i), "GPUMultislice": ([_i, _i, _f], _i),
    "GetResult": ([_i, _i, _fp, _i], _i), "GetAvgResult": ([_i, _i, _fp, _fp, _i], _i),
    "ClearDetMem_h": ([_i], _i), "ClearDetMem_d": ([], _i), "Cleanup": ([], _i), "FreeLibMem": ([], None),
    "JMS_SetStream": ([_p], _i),
    "JMS_ScanGPU": ([_i, _fp, _f, _i, _ip, _fp, _fp, _i], _i),
    "JMS_ScanGPUDevice": ([_i, _p, _f, _i, _ip, _p, _p, _i], _i),
    "JMS_SetScanBatch": ([_i], _i), "JMS_KernelLaunches": ([], C.c_longlong), "JMS_SetPassFusion": ([_i], _i),
    "JMS_ScanMultiFidelityDevice": ([_i, _i, _i, _p, _f, _i, _ip, _p], _i),
    "JMS_ScanMultiFidelity": ([_i, _i, _i, _fp, _f, _i, _ip, _fp], _i),
    "JMS_GridSupported": ([_i, _i], _i),
    "JMS_SetPrecision": ([_i], _i), "JMS_GetPrecision": ([], _i), "JMS_TcStatus": ([], _i),
    "JMS_TcLaunches": ([], C.c_longlong),
    "JMS_ReadoutDetAvg": ([_i, _i, _fp, _fp], _i),
    "JMS_CreateContext": ([], _i), "JMS_SelectContext": ([_i], _i), "JMS_DestroyContext": ([_i], _i),
    "JMS_GraphBegin": ([_i, _ip], _i), "JMS_GraphEnd": ([], _i), "JMS_GraphLaunch": ([_i, _p, _i], _i),
    "JMS_GraphDestroy": ([_i], _i),
    "JMS_NnConvForward": ([_p, _p, _p, _p, _i, _i, _i, _i, _i, _i, _p], _i),
    "JMS_NnConvBackward": ([_p, _p, _p, _p, _p, _p, _p, _i, _i, _i, _i, _i, _i, _p], _i),
    "JMS_NnPoolLinearForward": ([_p, _p, _p, _p, _i, _i, _i, _i, _p], _i),
    "JMS_NnPoolLinearBackward": ([_p, _p, _p, _p, _p, _p, _i, _i, _i, _i, _p], _i),
    "JMS_NnMseLoss": ([_p, _p, _p, _p, _i, _p], _i),
    "JMS_NnAdam": ([_p, _p, _p, _p, _p, _i, _f, _f, _f, _f, _i, _p], _i),
    "JMS_NnCastBf16": ([_p, _p, C.c_longlong, _p], _i),
    "JMS_NnPatches": ([_p, _i, _i, _i, _i, _p, _i, _p, _i, _p, _i, _i, _i, _i, _p, _p], _i),
    "JMS_SliReadHeader": ([C.c_char_p, C.POINTER(JMSSliHeader)], _i),
    "JMS_SliReadData": ([C.c_char_p, _fp], _i),
    "JMS_SliWrite": ([C.c_char_p, C.POINTER(JMSSliHeader), _fp], _i),
    "JMS_SliLoadSlice": ([C.c_char_p, _i], _i),
    "JMS_PgrSetup": ([_i, _i, _f, _f, _f, _i, _i, _i], _i),
    "JMS_PgrSetFormFactors": ([_i, _i, _f, _fp, _fp], _i),
    "JMS_PgrSetStream": ([_p], _i),
    "JMS_PgrCalculate": ([_i, _fp, _f, _i, C.c_ulonglong, _i, _i, _fp], _i),
    "JMS_ReadoutDetectorsNoAlloc": ([_p, _i, _p, _p], _i),
    "JMS_Autotune": ([_i, _i, _fp, _fp, _ip, _ip], _i),
    "JMS_SelectPlans": ([_i, _i], _i),
    "JMS_PlanCount": ([_i], _i),
    "JMS_PlanName": ([_i, C.c_char_p, _i], _i),
    "JMS_SetPassTiming": ([_i], None),
    "JMS_PassTiming": ([_dp, C.POINTER(C.c_longlong), _dp, C.POINTER(C.c_longlong)], _i),
}

_lib = None


def lib():
    """Loads libjms_b200.so; raises when it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m jmultislicelib_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def _fptr(a):
    return a.ctypes.data_as(_fp)


def _c64(a):
    return np.ascontiguousarray(a, np.complex64)


def sli_read(path):
    """EMS slice file -> (header dict, gratings complex64 [nvar, ny, nx]) (JMS_SliReadHeader / ReadData)."""
    h = JMSSliHeader()
    e = lib().JMS_SliReadHeader(os.fsencode(path), C.byref(h))
    if e:
        raise OSError(f"JMS_SliReadHeader({path}) returned {e}")
    d = {k: getattr(h, k) for k, _ in JMSSliHeader._fields_}
    d["title"] = h.title.decode("latin-1").rstrip("\x00 ")
    pgr = np.zeros((h.nvar, h.ny, h.nx), np.complex64)
    e = lib().JMS_SliReadData(os.fsencode(path), _fptr(pgr))
    if e:
        raise OSError(f"JMS_SliReadData({path}) returned {e}")
    return d, pgr


def sli_write(path, pgr, thickness, ekv, sx, sy, title="", content=0):
    """Writes gratings [nvar, ny, nx] as an EMS slice file (JMS_SliWrite)."""
    g = np.ascontiguousarray(pgr, np.complex64)
    if g.ndim == 2:
        g = g[None]
    h = JMSSliHeader(nx=g.shape[2], ny=g.shape[1], nvar=g.shape[0], content=content, thickness=thickness, ekv=ekv,
                     sx=sx, sy=sy)
    h.title = title.encode("latin-1")[:40]
    return lib().JMS_SliWrite(os.fsencode(path), C.byref(h), _fptr(g))


class JMS:
    """Python view of the library instance behind the flat C ABI.

    Method names and arguments follow CJMultiSlice (src/JMultiSlice.h) with
    numpy arrays in place of raw pointers; return codes are the library's.
    """

    def __init__(self):
        self.L = lib()
        self.nx = self.ny = 0

    # physics / grid
    def set_high_tension(self, kv):
        self.L.SetHighTension(kv)
        return self.L.GetWaveLength()

    def set_grid(self, nx, ny, a, b, c):
        self.L.SetGridSize(nx, ny)
        self.L.SetSupercellSizeABC(a, b, c)
        self.nx, self.ny = nx, ny

    def seed(self, s):
        self.L.SeedRngEx(s)

    # generators
    def calc_probe(self, alpha, alpha_rs=0.03, x0=0.0, y0=0.0, asym=0.0, adir=0.0, btx=0.0, bty=0.0, abrr=None):
        ab = np.zeros(48, np.float32) if abrr is None else np.ascontiguousarray(abrr, np.float32)
        prm = JMSProbeParams(m_wl=0.0, m_alpha=alpha, m_alpha_rs=alpha_rs, m_alpha_x0=x0, m_alpha_y0=y0,
                             m_alpha_asym=asym, m_alpha_adir=adir, m_btx=btx, m_bty=bty, m_abrr_coeff=_fptr(ab))
        wav = np.zeros((self.ny, self.nx), np.complex64)
        e = self.L.CalculateProbeWaveFourier(C.byref(prm), _fptr(wav))
        assert e == 0, e
        return wav

    def calc_propagator(self, fthick, otx=0.0, oty=0.0, ntype=0):
        pro = np.zeros((self.ny, self.nx), np.complex64)
        assert self.L.CalculatePropagator(fthick, otx, oty, _fptr(pro), ntype) == 0
        return pro

    def calc_ring_detector(self, beta0, beta1, phi0=0.0, phi1=0.0, th0x=0.0, th0y=0.0, kmom1=0, profile=b""):
        det = np.zeros((self.ny, self.nx), np.float32)
        msk = np.zeros(self.nx * self.ny, np.int32)
        ml = C.c_int(0)
        assert self.L.CalculateRingDetector(beta0, beta1, phi0, phi1, th0x, th0y, profile, _fptr(det),
                                            C.byref(ml), msk.ctypes.data_as(_ip), kmom1) == 0
        return det, msk[: ml.value].copy()

    # setup chain
    def setup(self, code, nslcvar, objslc, proidx, ndetper, ndet, imagedet, npg=None):
        nslcvar = np.ascontiguousarray(nslcvar, np.int32)
        objslc = np.ascontiguousarray(objslc, np.int32)
        proidx = np.ascontiguousarray(proidx, np.int32)
        npgx, npgy = (self.nx, self.ny) if npg is None else npg
        L = self.L
        e = [L.PhaseGratingSetup(code, npgx, npgy, len(nslcvar), int(nslcvar.max()), nslcvar.ctypes.data_as(_ip)),
             L.ObjectSliceSetup(len(objslc), objslc.ctypes.data_as(_ip)),
             L.PropagatorSetup(code, int(proidx.max()) + 1, proidx.ctypes.data_as(_ip)),
             L.DetectorSetup(code, ndetper, ndet, imagedet, 1)]
        return e

    def set_phase_grating(self, code, islc, pgr):
        pgr = _c64(pgr)
        nvar = pgr.shape[0] if pgr.ndim == 3 else 1
        return self.L.SetSlicePhaseGratings(code, islc, nvar, _fptr(pgr))

    def set_propagator(self, code, ipro, pro):
        return self.L.SetPropagatorData(code, ipro, _fptr(_c64(pro)))

    def set_detector(self, code, idet, det, msk=None):
        det = np.ascontiguousarray(det, np.float32)
        if msk is None or len(msk) == 0:
            return self.L.SetDetectorData(code, idet, _fptr(det), 0, None)
        msk = np.ascontiguousarray(msk, np.int32)
        return self.L.SetDetectorData(code, idet, _fptr(det), len(msk), msk.ctypes.data_as(_ip))

    def init_core(self, code):
        return self.L.InitCore(code, 1)

    def set_incident_wave(self, code, wav):
        return self.L.SetIncidentWave(code, _fptr(_c64(wav)))

    def set_phaseplate(self, code, ppl):
        return self.L.SetIncidentWavePhaseplate(code, _fptr(np.ascontiguousarray(ppl, np.float32)), 0)

    def offset(self, code, dx, dy, dz=0.0, ithread=0, ibtx=0, ibty=0):
        return self.L.OffsetIncomingWave(code, dx, dy, dz, ithread, ibtx, ibty)

    def gpu_multislice(self, islc0=0, accmode=0, weight=1.0):
        return self.L.GPUMultislice(islc0, accmode, weight)

    def num_det_planes(self):
        return self.L.GetDetetionSliceNum()

    def get_result(self, code, which, count, dtype=np.float32):
        dst = np.zeros(count, dtype)
        self.L.GetResult(code, which, dst.view(np.float32).ctypes.data_as(_fp), 0)
        return dst

    def get_avg_result(self, code, which, count, dtype=np.float32):
        dst = np.zeros(count, dtype)
        w = C.c_float(0)
        self.L.GetAvgResult(code, which, dst.view(np.float32).ctypes.data_as(_fp), C.byref(w), 0)
        return dst, w.value

    def readout_det_avg(self, which, count):
        """CJMultiSlice::ReadoutDetAvg on the device: (error, dst, weight)."""
        dst = np.zeros(count, np.float32)
        w = C.c_float(0)
        e = self.L.JMS_ReadoutDetAvg(CODE_GPU, which, _fptr(dst), C.byref(w))
        return e, dst, w.value

    def unscramble_hash(self):
        out = np.zeros(self.nx * self.ny, np.uint32)
        self.L.GetUnscrambleHash(out.ctypes.data_as(C.POINTER(C.c_uint)))
        return out

    def cleanup(self):
        return self.L.Cleanup()

    # additions
    def set_precision(self, mode):
        """0 = FP32 passes, 1 = tensor-core passes with BF16 hi+lo operands, 2 = with FP16 hi+lo (JMS_SetPrecision)."""
        return self.L.JMS_SetPrecision(int(mode))

    def tc_status(self):
        """0, or 1 if a tensor-core pass gave up waiting for its matrix products (JMS_TcStatus)."""
        return self.L.JMS_TcStatus()

    def set_stream(self, stream_ptr):
        return self.L.JMS_SetStream(C.c_void_p(stream_ptr))

    def sli_load_slice(self, path, islc):
        return self.L.JMS_SliLoadSlice(os.fsencode(path), islc)

    # ---- on-device phase gratings (CJEElaSca, src/JEElaSca.h:98-273)
    def pgr_setup(self, nx, ny, a, b, ekv, thermal=0, bwl_pot=0, bwl_pgr=1):
        self.pgr_grid = (nx, ny)
        return self.L.JMS_PgrSetup(nx, ny, a, b, ekv, thermal, bwl_pot, bwl_pgr)

    def pgr_set_form_factors(self, ff, sk, biso=None):
        ff = _c64(ff)
        bi = None if biso is None else np.ascontiguousarray(biso, np.float32)
        return self.L.JMS_PgrSetFormFactors(ff.shape[0], ff.shape[1], sk, _fptr(ff), None if bi is None else _fptr(bi))

    def pgr_set_stream(self, stream_ptr):
        """Stream of the generator's kernels (0 / None: the context's stream)."""
        return self.L.JMS_PgrSetStream(C.c_void_p(stream_ptr or None))

    def pgr_calculate(self, atoms, cz, ngr=1, seed=0, islc=-1, ivar0=0, want=True):
        """atoms [natom, 5]: fractional x, y, z, occupancy, type.  Returns
        (error, gratings complex64 [ngr, ny, nx] or None)."""
        at = np.ascontiguousarray(atoms, np.float32).reshape(-1, 5)
        nx, ny = self.pgr_grid
        out = np.zeros((ngr, ny, nx), np.complex64) if want else None
        e = self.L.JMS_PgrCalculate(at.shape[0], _fptr(at), cz, ngr, seed, islc, ivar0,
                                    None if out is None else _fptr(out))
        return e, out

    def scan(self, pos, npass, dz=0.0, varseq=None, ndetslc=None, ndet=None, bin=0):
        pos = np.ascontiguousarray(pos, np.float32)
        npos = pos.shape[0]
        nd = self.L.GetDetetionSliceNum() if ndetslc is None else ndetslc
        ndt = self.L.GetDetNum() if ndet is None else ndet
        out = np.zeros((npos, nd, ndt), np.float32)
        vs = None if varseq is None else np.ascontiguousarray(varseq, np.int32)
        ob = np.zeros((npos, self.ny // bin, self.nx // bin), np.float32) if bin else None
        e = self.L.JMS_ScanGPU(npos, _fptr(pos), dz, npass, None if vs is None else vs.ctypes.data_as(_ip),
                               _fptr(out), None if ob is None else _fptr(ob), bin)
        return e, out, ob
