"""Library contexts (one setup per grid size, each on its own stream), their
concurrent scans, and CUDA-graph capture and replay of those scans."""
import numpy as np
import pytest

from tests import golden_cases as G
from tests import product_cases as PC

pytestmark = pytest.mark.gpu
GPU = 2
TOL = 1e-4


@pytest.fixture(scope="module")
def J():
    import jmultislicelib_b200 as jb

    j = jb.JMS()
    yield j
    j.L.JMS_SelectContext(0)


def _scan_setup(J, nx, ny, nobj, nvar, seed):
    """Synthetic specimen on an nx x ny grid in the selected context."""
    a, b = 0.045 * nx, 0.045 * ny
    J.cleanup()
    J.set_high_tension(300.0)
    J.set_grid(nx, ny, a, b, 0.4)
    pro = J.calc_propagator(0.19525, 0.0, 0.0, 1)
    dets = [J.calc_ring_detector(b0, b1) for (b0, b1) in ((0, 10), (20, 50), (80, 200))]
    probe = J.calc_probe(22.0)
    pgr = PC.synthetic_specimen(nx, ny, 2, nvar, seed)
    objslc = np.arange(nobj) % 2
    assert J.setup(GPU, [nvar, nvar], objslc, [0, 0], max(nobj // 4, 1), 3, G.INT) == [0, 0, 0, 0]
    for s in range(2):
        assert J.set_phase_grating(GPU, s, pgr[s]) == 0
    assert J.set_propagator(GPU, 0, pro) == 0
    for i, (d, m) in enumerate(dets):
        assert J.set_detector(GPU, i, d, m) == 0
    assert J.init_core(GPU) == 0
    assert J.set_incident_wave(GPU, probe) == 0
    rng = np.random.default_rng(seed)
    pos = rng.uniform(0, min(a, b), (9, 2)).astype(np.float32)
    from oracle import oracle as OR

    orng = OR.Rng(seed)
    varseq = np.stack([orng.variant_sequence([nvar, nvar], objslc) for _ in range(2)])
    return pos, varseq


def _scan_device(J, pos, varseq, npass, d_out):
    import ctypes as C

    import torch

    d_pos = torch.from_numpy(pos).cuda()
    torch.cuda.synchronize()   # the library stream does not wait for torch's
    vs = np.ascontiguousarray(varseq, np.int32)
    e = J.L.JMS_ScanGPUDevice(len(pos), d_pos.data_ptr(), 0.0, npass, vs.ctypes.data_as(C.POINTER(C.c_int)),
                              d_out.data_ptr(), None, 0)
    return e, d_pos


def test_contexts_hold_independent_setups(J):
    ids = [J.L.JMS_CreateContext(), J.L.JMS_CreateContext()]
    assert ids[0] > 0 and ids[1] > ids[0]
    try:
        cases = {ids[0]: "msa", ids[1]: "msb"}
        for cid, name in cases.items():
            assert J.L.JMS_SelectContext(cid) >= 0
            PC.setup_case(J, G.case(name))
        for cid, name in cases.items():   # run after both setups exist
            J.L.JMS_SelectContext(cid)
            c = G.case(name)
            J.nx, J.ny = c["nx"], c["ny"]
            J.seed(c["seed"])
            for (dx, dy, dz, ibtx, ibty, accmode, w) in c["runs"]:
                assert J.offset(GPU, float(dx), float(dy), float(dz), 0, int(ibtx), int(ibty)) == 0
                assert J.gpu_multislice(c["islc0"], int(accmode), float(w)) == 0
            nd = J.num_det_planes()
            di = J.get_result(GPU, G.INT, nd * c["ndet"]).reshape(nd, c["ndet"])
            assert G.rel_err(di, c["det_int"]) < TOL, name
    finally:
        J.L.JMS_SelectContext(0)
        for cid in ids:
            assert J.L.JMS_DestroyContext(cid) == 0
    assert J.L.JMS_SelectContext(ids[0]) == -1
    assert J.L.JMS_DestroyContext(0) == 1


def test_uneven_scans_run_concurrently_and_replay_as_a_graph(J):
    import ctypes as C

    import torch

    grids = [(256, 256, 12, 3), (384, 384, 8, 2), (128, 96, 16, 4)]
    ids, setups, outs = [], [], []
    try:
        for k, (nx, ny, nobj, nvar) in enumerate(grids):
            cid = J.L.JMS_CreateContext()
            ids.append(cid)
            J.L.JMS_SelectContext(cid)
            setups.append(_scan_setup(J, nx, ny, nobj, nvar, seed=40 + k))
        # sequential runs, one context after the other
        seq = []
        for cid, (pos, vs) in zip(ids, setups):
            J.L.JMS_SelectContext(cid)
            nd, ndet = J.num_det_planes(), 3
            d = torch.zeros((len(pos), nd, ndet), dtype=torch.float64, device="cuda")
            torch.cuda.synchronize()   # the contexts work on their own streams
            e, _ = _scan_device(J, pos, vs, 2, d)
            assert e == 0
            torch.cuda.synchronize()
            seq.append(d.cpu().numpy())
        # all three enqueued back to back (each on its context's stream)
        keep = []
        for cid, (pos, vs) in zip(ids, setups):
            J.L.JMS_SelectContext(cid)
            outs.append(torch.zeros((len(pos), J.num_det_planes(), 3), dtype=torch.float64, device="cuda"))
            keep.append(torch.from_numpy(pos).cuda())
        torch.cuda.synchronize()
        for cid, (pos, vs), d, dp in zip(ids, setups, outs, keep):
            J.L.JMS_SelectContext(cid)
            vsa = np.ascontiguousarray(vs, np.int32)
            assert J.L.JMS_ScanGPUDevice(len(pos), dp.data_ptr(), 0.0, 2, vsa.ctypes.data_as(C.POINTER(C.c_int)),
                                         d.data_ptr(), None, 0) == 0
        torch.cuda.synchronize()
        for a, b in zip(outs, seq):
            np.testing.assert_array_equal(a.cpu().numpy(), b)
        # the same three scans captured into one graph and replayed twice
        for d in outs:
            d.zero_()
        torch.cuda.synchronize()
        arr = np.array(ids, np.int32)
        assert J.L.JMS_GraphBegin(len(ids), arr.ctypes.data_as(C.POINTER(C.c_int))) == 0
        for cid, (pos, vs), d, dp in zip(ids, setups, outs, keep):
            J.L.JMS_SelectContext(cid)
            vsa = np.ascontiguousarray(vs, np.int32)
            assert J.L.JMS_ScanGPUDevice(len(pos), dp.data_ptr(), 0.0, 2, vsa.ctypes.data_as(C.POINTER(C.c_int)),
                                         d.data_ptr(), None, 0) == 0
        h = J.L.JMS_GraphEnd()
        assert h >= 1
        try:
            for rep in range(2):
                for d in outs:
                    d.zero_()
                torch.cuda.synchronize()
                assert J.L.JMS_GraphLaunch(h, None, 1) == 0
                for a, b in zip(outs, seq):
                    np.testing.assert_array_equal(a.cpu().numpy(), b)
        finally:
            assert J.L.JMS_GraphDestroy(h) == 0
    finally:
        J.L.JMS_SelectContext(0)
        for cid in ids:
            J.L.JMS_DestroyContext(cid)
