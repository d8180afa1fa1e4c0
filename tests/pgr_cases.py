"""Helpers for the phase-grating generator tests.

``golden(name)`` reads one case of tests/golden/ref_pgr.npz (the reference's
CJEElaSca gratings, tests/golden/make_golden_pgr.py).  ``sites`` and
``qep_positions`` restate on the host what the generator does before its
kernels: site linking (CStructure::SetAtomSites, src/Structure.cpp:441-491)
and the QEP displacement draws (SplitMix64 stream of the seed, Box-Muller),
so the FP64 oracle can be given the same atom positions.
"""
from __future__ import annotations

import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_pgr.npz")
CASES = ("g0", "g1", "g2")
_cache = None


def golden(name: str) -> dict:
    global _cache
    if _cache is None:
        with np.load(GOLDEN) as z:
            _cache = {k: z[k] for k in z.files}
    pre = name + "_"
    d = {k[len(pre):]: v for k, v in _cache.items() if k.startswith(pre)}
    for k in ("nx", "ny", "thermal", "absorb"):
        d[k] = int(d[k])
    for k in ("a", "b", "c", "abf", "sk", "wl"):
        d[k] = float(d[k])
    return d


def atoms_array(pos, occ, atype):
    """[natom, 5] rows: fractional x, y, z, occupancy, type."""
    pos = np.asarray(pos, np.float32).reshape(-1, 3)
    return np.column_stack([pos, np.asarray(occ, np.float32), np.asarray(atype, np.float32)]).astype(np.float32)


def type_biso(atype, biso_per_atom, ntype):
    out = np.zeros(ntype, np.float32)
    for t, b in zip(atype, biso_per_atom):
        out[int(t)] = b
    return out


def sites(atoms, a, b, cz, tbiso, thermal):
    """Site linking as the generator does it; returns (site_of_atom,
    base [nsite, 2] fractional, u_frac [nsite, 2])."""
    site_pos, site_atoms = [], []
    site_of = np.zeros(len(atoms), np.int64)
    for i, r in enumerate(atoms):
        found = -1
        for s, p in enumerate(site_pos):
            d = np.sqrt(((r[0] - p[0]) * a) ** 2 + ((r[1] - p[1]) * b) ** 2 + ((r[2] - p[2]) * cz) ** 2)
            if d < 0.05:
                found = s
                break
        if found < 0:
            site_pos.append([float(r[0]), float(r[1]), float(r[2])])
            site_atoms.append([i])
            site_of[i] = len(site_pos) - 1
            continue
        site_atoms[found].append(i)
        o = sum(float(atoms[k][3]) for k in site_atoms[found])
        if o > 0:
            site_pos[found] = [sum(float(atoms[k][c]) * float(atoms[k][3]) for k in site_atoms[found]) / o
                               for c in range(3)]
        site_of[i] = found
    base = np.array([[p[0], p[1]] for p in site_pos], np.float64)
    u = np.zeros((len(site_pos), 2))
    if thermal == 2:
        for s, ats in enumerate(site_atoms):
            o = sum(float(atoms[k][3]) for k in ats)
            bs = sum(float(tbiso[int(atoms[k][4])]) * float(atoms[k][3]) for k in ats) / o if o > 0 else 0.0
            if bs > 0:
                us = np.sqrt(bs) / np.sqrt(8.0 * np.pi ** 2)
                u[s] = (us / a, us / b)
    return site_of, base, u


_GAMMA = np.uint64(0x9E3779B97F4A7C15)


def _sm64(seed: int, k: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + k.astype(np.uint64) * _GAMMA
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def qep_positions(base, u, ngr, seed):
    """[ngr, nsite, 2] fractional site positions of ngr gratings."""
    nsite = base.shape[0]
    c = np.arange(ngr * nsite, dtype=np.uint64)
    u1 = ((_sm64(seed, 2 * c + np.uint64(1)) >> np.uint64(11)) + np.uint64(1)).astype(np.float64) * 2.0 ** -53
    u2 = (_sm64(seed, 2 * c + np.uint64(2)) >> np.uint64(11)).astype(np.float64) * 2.0 ** -53
    r = np.sqrt(-2.0 * np.log(u1))
    n1 = (r * np.cos(2 * np.pi * u2)).reshape(ngr, nsite)
    n2 = (r * np.sin(2 * np.pi * u2)).reshape(ngr, nsite)
    out = np.repeat(base[None], ngr, axis=0).copy()
    moving = (u[:, 0] != 0) | (u[:, 1] != 0)
    out[:, :, 0] += np.where(moving, u[:, 0] * n1, 0.0)
    out[:, :, 1] += np.where(moving, u[:, 1] * n2, 0.0)
    return out
