"""The allocation-free detector readout (JMS_ReadoutDetectorsNoAlloc).

It serves callers that cannot let the library allocate device memory while
they run; its scratch is a fixed device array inside the library.  This test
checks it, through the C ABI, against the library's regular path for the same
readout -- GPUMultislice started at the exit plane, which reads out the
incoming wave with the integrating detectors -- on two calls in a row with
different waves, and checks that a request larger than the fixed scratch is
refused.  It lives in its own file, collected last, so a failure here comes
after every other test has run.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-4
GPU = 2


def _setup(J, nx, ny, nobj):
    J.cleanup()
    J.set_high_tension(300.0)
    J.set_grid(nx, ny, 0.045 * nx, 0.045 * ny, 0.4)
    J.calc_propagator(0.19525, 0.0, 0.0, 1)
    dets = [J.calc_ring_detector(0, 10), J.calc_ring_detector(20, 50), J.calc_ring_detector(10, 60, kmom1=1)]
    objslc = np.arange(nobj) % 2
    assert J.setup(GPU, [1, 1], objslc, [0, 0], 2, len(dets) + 1, 1) == [0, 0, 0, 0]
    for s in range(2):
        assert J.set_phase_grating(GPU, s, np.ones((1, ny, nx), np.complex64)) == 0
    assert J.set_propagator(GPU, 0, np.ones((ny, nx), np.complex64)) == 0
    for i, (d, m) in enumerate(dets):
        assert J.set_detector(GPU, i, d, m) == 0
    # a fourth detector without a mask: a smooth weight over the whole grid
    ky, kx = np.meshgrid(np.fft.fftfreq(ny), np.fft.fftfreq(nx), indexing="ij")
    assert J.set_detector(GPU, len(dets), (1.0 + 0.5 * np.cos(2 * np.pi * (kx + ky))).astype(np.float32)) == 0
    assert J.init_core(GPU) == 0
    return len(dets) + 1


def _regular_readout(J, wav, nobj, ndet):
    """Integrated detectors of wav via GPUMultislice(islc0 = nobjslc)."""
    assert J.L.SetIncomingWaveGPU(wav.view(np.float32).ctypes.data_as(C.POINTER(C.c_float)), 0) == 0
    assert J.gpu_multislice(nobj, 0, 1.0) == 0
    nd = J.num_det_planes()
    return J.get_result(GPU, 1, nd * ndet).reshape(nd, ndet)[-1].astype(np.float64)


def test_no_alloc_readout_matches_regular_path_twice():
    import torch

    import jmultislicelib_b200 as jb

    J = jb.JMS()
    nx, ny, nobj = 128, 96, 4
    ndet = _setup(J, nx, ny, nobj)
    rng = np.random.default_rng(5)
    out = torch.zeros(ndet, dtype=torch.float64, device="cuda")
    for call in range(2):
        wav = (rng.normal(size=(ny, nx)) + 1j * rng.normal(size=(ny, nx))).astype(np.complex64)
        wav /= np.sqrt((np.abs(wav) ** 2).sum())
        expect = _regular_readout(J, wav, nobj, ndet)
        d_wav = torch.from_numpy(wav.view(np.float32).copy()).cuda()
        torch.cuda.synchronize()
        e = J.L.JMS_ReadoutDetectorsNoAlloc(d_wav.data_ptr(), 1, out.data_ptr(), None)
        torch.cuda.synchronize()
        assert e == 0, e
        got = out.cpu().numpy()
        rel = np.abs(got - expect) / np.maximum(np.abs(expect), 1e-30)
        assert rel.max() < TOL, (call, got, expect)


def test_no_alloc_readout_on_a_caller_stream():
    """The wave is written on a stream of the caller's and the readout is
    enqueued on that stream: the result must follow the write, twice."""
    import torch

    import jmultislicelib_b200 as jb

    J = jb.JMS()
    nx, ny, nobj = 128, 96, 4
    ndet = _setup(J, nx, ny, nobj)
    rng = np.random.default_rng(6)
    s = torch.cuda.Stream()
    out = torch.zeros(ndet, dtype=torch.float64, device="cuda")
    d_wav = torch.zeros(2 * nx * ny, dtype=torch.float32, device="cuda")
    for call in range(2):
        wav = (rng.normal(size=(ny, nx)) + 1j * rng.normal(size=(ny, nx))).astype(np.complex64)
        wav /= np.sqrt((np.abs(wav) ** 2).sum())
        expect = _regular_readout(J, wav, nobj, ndet)
        h_wav = torch.from_numpy(wav.view(np.float32).ravel().copy()).pin_memory()
        torch.cuda.synchronize()
        with torch.cuda.stream(s):
            d_wav.copy_(h_wav, non_blocking=True)     # the wave arrives on the caller's stream
            e = J.L.JMS_ReadoutDetectorsNoAlloc(d_wav.data_ptr(), 1, out.data_ptr(), C.c_void_p(s.cuda_stream))
            got_d = out.clone()
        s.synchronize()
        assert e == 0, e
        got = got_d.cpu().numpy()
        rel = np.abs(got - expect) / np.maximum(np.abs(expect), 1e-30)
        assert rel.max() < TOL, (call, got, expect)


def test_no_alloc_readout_refuses_oversize_request():
    import torch

    import jmultislicelib_b200 as jb

    J = jb.JMS()
    nx, ny, nobj = 128, 96, 4
    ndet = _setup(J, nx, ny, nobj)
    nblk = (ny + 7) // 8
    nwave = 65536 // (ndet * nblk) + 1           # one wave more than the scratch array holds
    d_wav = torch.zeros(2, dtype=torch.float32, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    assert J.L.JMS_ReadoutDetectorsNoAlloc(d_wav.data_ptr(), nwave, out.data_ptr(), None) == 131
