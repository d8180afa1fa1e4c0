"""On-device phase gratings (JMS_Pgr*, the counterpart of CJEElaSca's
CalculatePhasegratingGPU) against the reference's gratings and the FP64
oracle; gratings generated into the multislice setup run like uploaded ones."""
import numpy as np
import pytest

from tests import golden_cases as G
from tests import pgr_cases as PG

pytestmark = pytest.mark.gpu
GPU = 2
TOL_REF = 2e-5      # max |t - t_ref|: the reference forms phases and sums in FP32
TOL_FP64 = 5e-6     # max |t - t_fp64|


@pytest.fixture(scope="module")
def J():
    import jmultislicelib_b200 as jb

    return jb.JMS()


def _setup(J, c, thermal=None, bwl_pot=0, bwl_pgr=1):
    th = c["thermal"] if thermal is None else thermal
    assert J.pgr_setup(c["nx"], c["ny"], c["a"], c["b"], 300.0, th, bwl_pot, bwl_pgr) == 0
    tb = PG.type_biso(c["atype"], c["biso"], len(c["ff"]))
    assert J.pgr_set_form_factors(c["ff"], c["sk"], tb) == 0
    return PG.atoms_array(c["pos"], c["occ"], c["atype"]), tb


def _oracle(c, atoms, positions, bwl_pot=0, bwl_pgr=1):
    from oracle import oracle as OR

    return OR.pgr(c["nx"], c["ny"], c["a"], c["b"], c["wl"], positions, c["occ"], c["atype"], c["ff"], c["sk"],
                  bwl_pot=bwl_pot, bwl_pgr=bwl_pgr)


@pytest.mark.parametrize("name", PG.CASES)
def test_pgr_matches_reference_and_fp64(J, name):
    c = PG.golden(name)
    atoms, tb = _setup(J, c)
    e, t = J.pgr_calculate(atoms, c["c"])
    assert e == 0
    assert np.abs(t[0] - c["pgr"]).max() < TOL_REF
    site_of, base, _ = PG.sites(atoms, c["a"], c["b"], c["c"], tb, c["thermal"])
    assert np.abs(t[0] - _oracle(c, atoms, base[site_of])).max() < TOL_FP64


@pytest.mark.parametrize("bwl_pot,bwl_pgr", [(1, 1), (0, 0), (1, 0)])
def test_pgr_band_limit_switches(J, bwl_pot, bwl_pgr):
    c = PG.golden("g1")
    atoms, tb = _setup(J, c, bwl_pot=bwl_pot, bwl_pgr=bwl_pgr)
    e, t = J.pgr_calculate(atoms, c["c"])
    assert e == 0
    site_of, base, _ = PG.sites(atoms, c["a"], c["b"], c["c"], tb, 0)
    o = _oracle(c, atoms, base[site_of], bwl_pot=bwl_pot, bwl_pgr=bwl_pgr)
    assert np.abs(t[0] - o).max() < TOL_FP64


@pytest.mark.parametrize("nx,ny", [(64, 96), (80, 120), (40, 80)])
def test_pgr_grid_shapes(J, nx, ny):
    """Non-square grids whose width and half height are not multiples of the
    synthesis tile: the rows summed directly, their mirrors (ny - iy,
    (nx - ix) mod nx) and the Nyquist row and column all against the FP64
    oracle.  The shapes keep every pixel at least 1e-4 (relative) away from the
    2/3 band-limit radius on this cell: on a pixel exactly at that radius (80 x
    48, 96 x 48 here) the aperture's float comparison, which follows the
    reference, and the oracle's double comparison may disagree."""
    c = dict(PG.golden("g1"), nx=nx, ny=ny)
    atoms, tb = _setup(J, c)
    e, t = J.pgr_calculate(atoms, c["c"])
    assert e == 0
    site_of, base, _ = PG.sites(atoms, c["a"], c["b"], c["c"], tb, c["thermal"])
    assert np.abs(t[0] - _oracle(c, atoms, base[site_of])).max() < TOL_FP64


def test_pgr_qep_draws(J):
    """Every grating of a QEP batch is the grating of its own displaced sites."""
    c = PG.golden("g2")
    atoms, tb = _setup(J, c, thermal=2)
    ngr, seed = 5, 987654321
    e, t = J.pgr_calculate(atoms, c["c"], ngr=ngr, seed=seed)
    assert e == 0
    site_of, base, u = PG.sites(atoms, c["a"], c["b"], c["c"], tb, 2)
    assert (u > 0).all()
    P = PG.qep_positions(base, u, ngr, seed)
    for g in range(ngr):
        assert np.abs(t[g] - _oracle(c, atoms, P[g][site_of])).max() < TOL_FP64, g
    assert np.abs(t[0] - t[1]).max() > 1e-3        # the draws differ
    e, t2 = J.pgr_calculate(atoms, c["c"], ngr=ngr, seed=seed)
    np.testing.assert_array_equal(t, t2)            # and repeat with the seed


def test_pgr_512_perovskite_slice(J):
    """The scan workload's size: 6x6 cells of a B + 2 O layer on 512^2."""
    from jmultislicelib_b200 import synthetic as S

    c = dict(PG.golden("g1"))
    sites = [(0, 0.5, 0.5, 1.0), (1, 0.5, 0.0, 1.0), (1, 0.0, 0.5, 1.0)]
    pos, occ, typ = [], [], []
    for i in range(6):
        for j in range(6):
            for (t_, fx, fy, o) in sites:
                pos.append(((i + fx) / 6, (j + fy) / 6, 0.0))
                occ.append(o)
                typ.append(t_)
    c.update(nx=512, ny=512, a=6 * S.A_CELL, b=6 * S.A_CELL, occ=np.array(occ, np.float32),
             atype=np.array(typ, np.int32), pos=np.array(pos, np.float32), thermal=0)
    # the g1 tables were sampled for a 96 x 64 grid; resample for 512^2 the same way
    assert J.pgr_setup(512, 512, c["a"], c["b"], 300.0, 0, 0, 1) == 0
    nk = 12 * 512
    sk = (512 / c["a"]) / nk
    q = np.arange(nk) * sk
    ff = np.stack([np.interp(q, np.arange(len(f)) * c["sk"], f.real, right=0.0)
                   + 1j * np.interp(q, np.arange(len(f)) * c["sk"], f.imag, right=0.0) for f in c["ff"]])
    assert J.pgr_set_form_factors(ff.astype(np.complex64), sk) == 0
    c.update(ff=ff.astype(np.complex64), sk=sk)
    atoms = PG.atoms_array(c["pos"], c["occ"], c["atype"])
    e, t = J.pgr_calculate(atoms, S.A_CELL / 2)
    assert e == 0
    o = _oracle(c, atoms, c["pos"][:, :2].astype(np.float64))
    assert np.abs(t[0] - o).max() < TOL_FP64


def test_pgr_into_multislice_setup(J):
    """Gratings generated into the grating store give the same multislice
    result as the same gratings uploaded with SetSlicePhaseGratings."""
    c = PG.golden("g0")
    nx, ny = c["nx"], c["ny"]
    atoms, tb = _setup(J, c, thermal=2)

    def run(upload):
        J.cleanup()
        J.set_high_tension(300.0)
        J.set_grid(nx, ny, c["a"], c["b"], c["c"])
        pro = J.calc_propagator(c["c"], 0.0, 0.0, 1)
        dets = [J.calc_ring_detector(b0, b1) for (b0, b1) in ((0, 10), (20, 50), (80, 200))]
        probe = J.calc_probe(25.0)
        objslc = np.arange(12) % 2
        assert J.setup(GPU, [3, 3], objslc, [0, 0], 4, 3, G.INT) == [0, 0, 0, 0]
        if upload is None:
            out = []
            for s in range(2):
                e, t = J.pgr_calculate(atoms, c["c"], ngr=3, seed=100 + s, islc=s, ivar0=0)
                assert e == 0
                out.append(t)
        else:
            for s in range(2):
                assert J.set_phase_grating(GPU, s, upload[s]) == 0
            out = upload
        assert J.set_propagator(GPU, 0, pro) == 0
        for i, (d, m) in enumerate(dets):
            assert J.set_detector(GPU, i, d, m) == 0
        assert J.init_core(GPU) == 0
        assert J.set_incident_wave(GPU, probe) == 0
        J.seed(77)
        assert J.offset(GPU, 0.3, 0.4, 0.0) == 0
        assert J.gpu_multislice(0, 0, 1.0) == 0
        nd = J.num_det_planes()
        return out, J.get_result(GPU, G.INT, nd * 3)

    gen, d_gen = run(None)
    _, d_up = run(gen)
    np.testing.assert_array_equal(d_gen, d_up)
    assert J.pgr_calculate(atoms, c["c"], ngr=4, seed=1, islc=0, ivar0=0, want=False)[0] == 9   # 4 > 3 variants
    J.cleanup()


def test_pgr_own_stream(J):
    """Gratings generated on a stream of the generator's own (JMS_PgrSetStream),
    ordered before the scan by an event, give the scan on the context's stream
    the same result as gratings generated on that stream itself."""
    import torch

    c = PG.golden("g0")
    nx, ny = c["nx"], c["ny"]
    atoms, tb = _setup(J, c, thermal=2)
    cs, gs = torch.cuda.Stream(), torch.cuda.Stream()
    objslc = np.arange(12) % 2
    pos = np.random.default_rng(3).uniform(0, c["a"], (5, 2)).astype(np.float32)
    varseq = np.stack([objslc * 0 + (k % 3) for k in range(2)]).astype(np.int32)

    def run(own):
        J.cleanup()
        J.set_stream(cs.cuda_stream)
        J.set_high_tension(300.0)
        J.set_grid(nx, ny, c["a"], c["b"], c["c"])
        pro = J.calc_propagator(c["c"], 0.0, 0.0, 1)
        dets = [J.calc_ring_detector(b0, b1) for (b0, b1) in ((0, 10), (20, 50), (80, 200))]
        assert J.setup(GPU, [3, 3], objslc, [0, 0], 4, 3, G.INT) == [0, 0, 0, 0]
        assert J.set_propagator(GPU, 0, pro) == 0
        for i, (d, m) in enumerate(dets):
            assert J.set_detector(GPU, i, d, m) == 0
        assert J.init_core(GPU) == 0
        assert J.set_incident_wave(GPU, J.calc_probe(25.0)) == 0
        torch.cuda.synchronize()
        if own:
            J.pgr_set_stream(gs.cuda_stream)
        for s in range(2):
            e, _ = J.pgr_calculate(atoms, c["c"], ngr=3, seed=100 + s, islc=s, ivar0=0, want=False)
            assert e == 0
        if own:
            ev = torch.cuda.Event()
            ev.record(gs)
            cs.wait_event(ev)
            J.pgr_set_stream(0)
        e, out, _ = J.scan(pos, 2, varseq=varseq)
        assert e == 0
        return out

    try:
        ref = run(False)
        np.testing.assert_array_equal(run(True), ref)
        assert np.abs(ref).max() > 0
    finally:
        J.pgr_set_stream(0)
        J.cleanup()
        J.set_stream(0)


def test_pgr_errors(J):
    c = PG.golden("g0")
    assert J.pgr_setup(100, 64, c["a"], c["b"], 300.0) == 8          # no line plan for 100
    atoms, _ = _setup(J, c)
    bad = atoms.copy()
    bad[0, 4] = 7
    assert J.pgr_calculate(bad, c["c"])[0] == 2
    assert J.pgr_calculate(atoms, c["c"], ngr=0, want=False)[0] == 3


def test_pgr_reproduces_synthetic_specimen(J):
    """With the workload's Gaussian form factors and no band limit, the
    generator reproduces the host-built specimen grating (no displacements)."""
    from jmultislicelib_b200 import synthetic as S

    nx = ny = 256
    a = b = 3 * S.A_CELL
    ff, sk = S.form_factor_tables(nx, ny, a, b, seed=11)
    assert J.pgr_setup(nx, ny, a, b, 300.0, 0, 0, 0) == 0
    assert J.pgr_set_form_factors(ff, sk) == 0
    amp, wid = S.atom_params(11)
    sig = S.interaction_constant(300.0)
    for layer in (0, 1):
        at = S.layer_atoms(3, 3, layer)
        e, t = J.pgr_calculate(at, S.DZ_SLICE)
        assert e == 0
        V = S.projected_potential(nx, ny, a, b, [(int(r[4]), r[0] * a, r[1] * b) for r in at], amp, wid)
        assert np.abs(t[0] - np.exp(1j * sig * V)).max() < 1e-6
