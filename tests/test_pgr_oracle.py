"""The FP64 oracle's phase-grating restatement against the reference's
CJEElaSca gratings (golden vectors), and the host-side helpers of the
generator tests."""
import numpy as np
import pytest

from tests import pgr_cases as PG


@pytest.mark.parametrize("name", PG.CASES)
def test_oracle_pgr_matches_reference(name):
    from oracle import oracle as OR

    c = PG.golden(name)
    atoms = PG.atoms_array(c["pos"], c["occ"], c["atype"])
    site_of, base, _ = PG.sites(atoms, c["a"], c["b"], c["c"], np.zeros(len(c["ff"])), 0)
    o = OR.pgr(c["nx"], c["ny"], c["a"], c["b"], c["wl"], base[site_of], c["occ"], c["atype"], c["ff"], c["sk"])
    # the reference forms translation phases and sums in FP32
    assert np.abs(o - c["pgr"]).max() < 2e-5
    assert abs(np.abs(o).mean() - np.abs(c["pgr"]).mean()) < 1e-6


def test_oracle_pgr_single_atom_is_centred():
    """One atom at the cell centre: the grating is symmetric about it."""
    from oracle import oracle as OR

    c = PG.golden("g0")
    n = 64
    o = OR.pgr(n, n, c["a"], c["b"], c["wl"], np.array([[0.5, 0.5]]), [1.0], [0], c["ff"][:1], c["sk"])
    ph = np.angle(o)
    assert np.unravel_index(np.argmax(ph), ph.shape) == (n // 2, n // 2)
    np.testing.assert_allclose(ph[n // 2, n // 2 + 5], ph[n // 2, n // 2 - 5], atol=1e-9)
    # no atoms: vacuum, t = 1 exactly
    v = OR.pgr(n, n, c["a"], c["b"], c["wl"], np.zeros((0, 2)), [], [], c["ff"][:1], c["sk"])
    np.testing.assert_allclose(v, 1.0, atol=1e-12)


def test_qep_draws_are_standard_normal():
    base = np.zeros((500, 2))
    u = np.ones((500, 2))
    p = PG.qep_positions(base, u, 200, seed=12345).reshape(-1, 2)
    assert abs(p.mean()) < 0.01
    assert abs(p.std() - 1.0) < 0.01
    assert abs(np.corrcoef(p[:, 0], p[:, 1])[0, 1]) < 0.01
    q = PG.qep_positions(base, u, 200, seed=12345).reshape(-1, 2)
    np.testing.assert_array_equal(p, q)


def test_sites_link_close_atoms():
    atoms = np.array([[0.0, 0.0, 0.0, 0.5, 0], [0.0, 0.0, 0.0, 0.5, 1], [0.5, 0.5, 0.0, 1.0, 2]], np.float32)
    site_of, base, u = PG.sites(atoms, 1.0, 1.0, 0.2, np.array([0.004, 0.006, 0.008]), 2)
    assert list(site_of) == [0, 0, 1]
    assert base.shape == (2, 2)
    # occupancy-weighted Biso of the mixed site: 0.005 nm^2
    np.testing.assert_allclose(u[0, 0], np.sqrt(0.005) / np.sqrt(8 * np.pi ** 2))
