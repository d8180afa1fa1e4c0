"""Multi-fidelity frozen-phonon scan (JMS_ScanMultiFidelity): a control-variate
estimate of the npass-configuration average from one full-grid pass and npass
passes of a coarser grid of the same specimen.

Checks, on a 3x3-cell ABO3 specimen (256^2 full grid, 128^2 coarse grid, 40
slices, 4 slice types x 4 phonon variants, 16 positions, 6 configurations):
- the estimate equals f(c0) - (g(c0) - mean_c g) assembled from separate
  JMS_ScanGPU runs of the two contexts (float rounding, 1e-6 of the largest
  signal per detector);
- for the 0-10 and 20-50 mrad detectors (inside the 128^2 band limit of
  72 mrad) the estimate is within 1e-4 of the full-grid 6-configuration
  average, which one full configuration alone misses by ~1e-3;
- the 80-200 mrad detector lies outside the coarse band limit (g = 0), so its
  estimate is the single full pass.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GPU = 2


@pytest.fixture(scope="module")
def pair():
    import jmultislicelib_b200 as jb
    from jmultislicelib_b200 import synthetic as S

    J = jb.JMS()
    base = dict(S.SCAN_512, ncell=3, nobj=40, nvar=4, nscan=4)
    lo = J.L.JMS_CreateContext()
    assert lo > 0
    for ctx, n in ((lo, 128), (0, 256)):
        J.L.JMS_SelectContext(ctx)
        cfg = dict(base, nx=n, ny=n)
        sp = S.make_specimen(n, n, cfg["ncell"], cfg["ncell"], cfg["nslice_types"], cfg["nvar"], cfg["seed"], cfg["kv"])
        _, _, _, _, pos = S.setup_library(J, cfg, specimen=sp)
    yield J, lo, pos, base
    J.L.JMS_SelectContext(0)
    J.L.JMS_DestroyContext(lo)


def _scan(J, ctx, pos, npass, varseq, nd, ndet):
    import ctypes as C

    J.L.JMS_SelectContext(ctx)
    out = np.zeros((len(pos), nd, ndet), np.float32)
    vs = np.ascontiguousarray(varseq, np.int32)
    e = J.L.JMS_ScanGPU(len(pos), pos.ctypes.data_as(C.POINTER(C.c_float)), 0.0, npass,
                        vs.ctypes.data_as(C.POINTER(C.c_int)), out.ctypes.data_as(C.POINTER(C.c_float)), None, 0)
    J.L.JMS_SelectContext(0)
    assert e == 0, e
    return out.astype(np.float64)


def test_multifidelity_estimate(pair):
    import ctypes as C

    J, lo, pos, cfg = pair
    pos = np.ascontiguousarray(pos, np.float32)
    nd, ndet = J.L.GetDetetionSliceNum(), J.L.GetDetNum()
    npass = 6
    varseq = np.random.default_rng(3).integers(0, cfg["nvar"], (npass, cfg["nobj"])).astype(np.int32)
    est = np.zeros((len(pos), nd, ndet), np.float32)
    e = J.L.JMS_ScanMultiFidelity(0, lo, len(pos), pos.ctypes.data_as(C.POINTER(C.c_float)), 0.0, npass,
                                  varseq.ctypes.data_as(C.POINTER(C.c_int)), est.ctypes.data_as(C.POINTER(C.c_float)))
    assert e == 0, e
    f0 = _scan(J, 0, pos, 1, varseq[:1], nd, ndet)
    g0 = _scan(J, lo, pos, 1, varseq[:1], nd, ndet)
    gm = _scan(J, lo, pos, npass, varseq, nd, ndet)
    plain = _scan(J, 0, pos, npass, varseq, nd, ndet)
    big = np.abs(plain).max(axis=(0, 1))
    ref = f0 - (g0 - gm)
    assert (np.abs(est - ref).max(axis=(0, 1)) / big < 1e-6).all()
    err = np.abs(est - plain).max(axis=(0, 1)) / big
    err_single = np.abs(f0 - plain).max(axis=(0, 1)) / big
    print("estimate vs plain", err, "single pass vs plain", err_single)
    assert err[0] < 1e-4 and err[1] < 1e-4, err
    assert err_single[0] > 10 * err[0] and err_single[1] > 10 * err[1], (err, err_single)
    # 80-200 mrad: outside the coarse grid's band, the estimate is the full pass of configuration 0
    assert np.abs(g0[..., 2]).max() == 0.0
    assert np.allclose(est[..., 2], f0[..., 2], rtol=1e-6, atol=0.0)


def test_multifidelity_rejects_mismatched_contexts(pair):
    import ctypes as C

    J, lo, pos, cfg = pair
    pos = np.ascontiguousarray(pos, np.float32)
    out = np.zeros((len(pos), 64), np.float32)
    vs = np.zeros((2, cfg["nobj"]), np.int32)
    # the same context twice, a missing context, and no variant sequence are refused
    assert J.L.JMS_ScanMultiFidelity(0, 0, len(pos), pos.ctypes.data_as(C.POINTER(C.c_float)), 0.0, 2,
                                     vs.ctypes.data_as(C.POINTER(C.c_int)), out.ctypes.data_as(C.POINTER(C.c_float))) == 1
    assert J.L.JMS_ScanMultiFidelity(0, 999, len(pos), pos.ctypes.data_as(C.POINTER(C.c_float)), 0.0, 2,
                                     vs.ctypes.data_as(C.POINTER(C.c_int)), out.ctypes.data_as(C.POINTER(C.c_float))) == 1
    assert J.L.JMS_ScanMultiFidelity(0, lo, len(pos), pos.ctypes.data_as(C.POINTER(C.c_float)), 0.0, 2,
                                     None, out.ctypes.data_as(C.POINTER(C.c_float))) == 1


def test_device_calls_back_to_back(pair):
    """Calls of JMS_ScanMultiFidelityDevice issued one after another without a
    host synchronisation (as a scan loop issues them) give the result of a lone
    call: each call's coarse stream waits for the full-grid stream before it
    clears the coarse scratch that the previous call's combine reads.  Two
    configurations make the full-grid pass the longer of the two streams, the
    order in which an unordered clear would zero the previous call's coarse
    sums before its combine."""
    import ctypes as C

    import torch

    J, lo, pos, cfg = pair
    pos = np.ascontiguousarray(pos, np.float32)
    nd, ndet = J.L.GetDetetionSliceNum(), J.L.GetDetNum()
    npass = 2
    varseq = np.random.default_rng(5).integers(0, cfg["nvar"], (npass, cfg["nobj"])).astype(np.int32)
    vs = varseq.ctypes.data_as(C.POINTER(C.c_int))
    d_pos = torch.from_numpy(pos).cuda()
    outs = [torch.zeros((len(pos), nd, ndet), dtype=torch.float64, device="cuda") for _ in range(7)]
    torch.cuda.synchronize()
    assert J.L.JMS_ScanMultiFidelityDevice(0, lo, len(pos), d_pos.data_ptr(), 0.0, npass, vs, outs[0].data_ptr()) == 0
    torch.cuda.synchronize()
    for o in outs[1:]:
        assert J.L.JMS_ScanMultiFidelityDevice(0, lo, len(pos), d_pos.data_ptr(), 0.0, npass, vs, o.data_ptr()) == 0
    torch.cuda.synchronize()
    ref = outs[0].cpu().numpy()
    assert np.abs(ref[..., 0]).max() > 0
    for k, o in enumerate(outs[1:]):
        assert np.array_equal(o.cpu().numpy(), ref), k
