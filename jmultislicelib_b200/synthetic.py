"""Seeded synthetic specimens and scan workloads (no public data is involved).

The benchmark workloads are defined on a cubic ABO3-like cell (a = 3.905 A;
sites A (0,0,0), B (1/2,1/2,1/2), O (1/2,1/2,0), (1/2,0,1/2), (0,1/2,1/2)),
sliced at z = 0 (A + O) and z = 1/2 (B + 2 O), each 1.9525 A thick.  Every
atom type has a projected potential V(r) = sum_i A_i exp(-r^2 / (2 w_i^2)),
i = 1, 2, with A_i ~ U(0.5, 5) V*A and w_i ~ U(0.1, 0.4) A drawn from the
workload seed (numpy PCG64).  Frozen-phonon variants displace every atom by
Gaussian noise of sigma 0.08 A in x and y.  The transmission function is
t = exp(i sigma V) with the relativistic interaction constant at the beam
energy; the phase is reduced modulo 2 pi in FP64 before the cast to
complex64.  Lengths handed to the library are in nm.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

A_CELL = 0.3905            # nm
DZ_SLICE = 0.19525         # nm
# CODATA 2018
_ME0, _QEL, _HPL, _C0 = 9.1093837015e-31, 1.602176634e-19, 6.62607015e-34, 299792458.0


def interaction_constant(kv: float) -> float:
    """sigma = 2 pi m e lambda / h^2 in rad / (V nm) (relativistic mass)."""
    e0 = _ME0 * _C0 ** 2 / _QEL / 1000.0              # keV
    lam = _C0 * _HPL / _QEL * 1.0e6 / np.sqrt(kv * (kv + 2 * e0)) * 1e-9   # m
    m = _ME0 * (1.0 + kv / e0)
    return 2 * np.pi * m * _QEL * lam / _HPL ** 2 * 1e-9


# fractional positions per slice type: (site type, fx, fy); types 0=A, 1=B, 2=O
LAYERS = {
    0: [(0, 0.0, 0.0), (2, 0.5, 0.5)],
    1: [(1, 0.5, 0.5), (2, 0.5, 0.0), (2, 0.0, 0.5)],
}


@dataclass
class Specimen:
    nx: int
    ny: int
    a: float                      # supercell edge x [nm]
    b: float                      # supercell edge y [nm]
    gratings: list = field(default_factory=list)   # per slice type: complex64 [nvar, ny, nx]
    layer_of_type: list = field(default_factory=list)
    potential: list = field(default_factory=list)  # per slice type: float64 [nvar, ny, nx] (V nm)


def atom_params(seed: int):
    rng = np.random.default_rng(seed)
    amp = rng.uniform(0.5, 5.0, (3, 2)) * 0.1    # V*A -> V*nm
    wid = rng.uniform(0.1, 0.4, (3, 2)) * 0.1    # A -> nm
    return amp, wid


def _gauss1d(coord, centres, width, period):
    d = coord[None, :] - centres[:, None]
    d = (d + 0.5 * period) % period - 0.5 * period
    return np.exp(-d * d / (2.0 * width[:, None] ** 2))


def projected_potential(nx, ny, a, b, atoms, amp, wid):
    """V(x, y) [V nm] on the grid as a sum of separable Gaussians (minimum image)."""
    x = np.arange(nx) * (a / nx)
    y = np.arange(ny) * (b / ny)
    cx, cy, ca, cw = [], [], [], []
    for (t, px, py) in atoms:
        for i in range(2):
            cx.append(px); cy.append(py); ca.append(amp[t, i]); cw.append(wid[t, i])
    cx, cy, ca, cw = map(np.asarray, (cx, cy, ca, cw))
    gx = _gauss1d(x, cx, cw, a)
    gy = _gauss1d(y, cy, cw, b)
    return (gy * ca[:, None]).T @ gx


def make_specimen(nx: int, ny: int, ncell_x: int, ncell_y: int, nslice_types: int, nvar: int, seed: int,
                  kv: float = 300.0, sigma_disp: float = 0.008, keep_potential: bool = False,
                  amp_scale: float = 1.0, wid_scale: float = 1.0) -> Specimen:
    """Specimen with nslice_types slice types (alternating A+O / B+2O layers,
    each with its own phonon draws) and nvar frozen-phonon variants per type.
    amp_scale and wid_scale multiply every atom's potential amplitudes and
    widths (1, 1: the workload's weak-phase cell; larger amplitudes and
    narrower atoms give a strongly scattering cell with the same geometry and
    phonon draws)."""
    amp, wid = atom_params(seed)
    amp = amp * amp_scale
    wid = wid * wid_scale
    rng = np.random.default_rng(seed + 1)
    a, b = ncell_x * A_CELL, ncell_y * A_CELL
    sig = interaction_constant(kv)
    sp = Specimen(nx=nx, ny=ny, a=a, b=b)
    for st in range(nslice_types):
        layer = LAYERS[st % 2]
        base = [(t, (ix + fx) * A_CELL, (iy + fy) * A_CELL)
                for iy in range(ncell_y) for ix in range(ncell_x) for (t, fx, fy) in layer]
        gr = np.empty((nvar, ny, nx), np.complex64)
        pots = []
        for v in range(nvar):
            d = rng.normal(0.0, sigma_disp, (len(base), 2)) if sigma_disp > 0 else np.zeros((len(base), 2))
            atoms = [(t, px + d[k, 0], py + d[k, 1]) for k, (t, px, py) in enumerate(base)]
            V = projected_potential(nx, ny, a, b, atoms, amp, wid)
            phase = np.mod(sig * V, 2 * np.pi)      # FP64 reduction before the complex64 cast
            gr[v] = np.exp(1j * phase).astype(np.complex64)
            if keep_potential:
                pots.append(V)
        sp.gratings.append(gr)
        sp.layer_of_type.append(st % 2)
        if keep_potential:
            sp.potential.append(np.asarray(pots))
    return sp


def scan_positions(nscan: int, x0: float, y0: float, extent: float) -> np.ndarray:
    """nscan x nscan raster [npos, 2] (dx, dy) in nm over one square of the given extent."""
    s = extent / nscan
    g = np.arange(nscan) * s
    xx, yy = np.meshgrid(x0 + g, y0 + g)
    return np.stack([xx.ravel(), yy.ravel()], axis=1).astype(np.float32)


# Workload of the headline metric: 6x6 cells on 512^2, 4 slice types (A+O,
# B+2O, A+O, B+2O with independent phonon draws), 16 variants each, 200
# slices, 300 kV, 22 mrad, Cs = 1 um, Fresnel propagator, annular detectors
# 0-10 / 20-50 / 80-200 mrad read every 20 slices, 64x64 raster over the unit
# cell in the middle of the supercell, 128x128 binned exit diffraction.
SCAN_512 = dict(nx=512, ny=512, ncell=6, nslice_types=4, nvar=16, nobj=200, kv=300.0, alpha=22.0, cs=1000.0,
                ntype=1, dets=((0.0, 10.0), (20.0, 50.0), (80.0, 200.0)), ndetper=20, nscan=64, bin=4,
                seed=20261204)
# single-probe point of the CPU-runnable case: 3x3 cells on 256^2, 2 slice
# types, 1 variant each, 100 slices, 25 mrad, aberration free, period 10
POINT_256 = dict(nx=256, ny=256, ncell=3, nslice_types=2, nvar=1, nobj=100, kv=300.0, alpha=25.0, cs=0.0,
                 ntype=1, dets=((0.0, 10.0), (20.0, 50.0), (80.0, 200.0)), ndetper=10, nscan=1, bin=0,
                 seed=20261203)


def setup_library(J, cfg: dict, specimen: Specimen | None = None):
    """Runs the reference setup chain on the library J for workload cfg.

    Returns (specimen, probe, propagator, detectors, positions)."""
    nx, ny = cfg["nx"], cfg["ny"]
    sp = specimen or make_specimen(nx, ny, cfg["ncell"], cfg["ncell"], cfg["nslice_types"], cfg["nvar"],
                                   cfg["seed"], cfg["kv"])
    J.cleanup()
    J.set_high_tension(cfg["kv"])
    J.set_grid(nx, ny, sp.a, sp.b, DZ_SLICE)
    pro = J.calc_propagator(DZ_SLICE, 0.0, 0.0, cfg["ntype"])
    dets = [J.calc_ring_detector(b0, b1) for (b0, b1) in cfg["dets"]]
    abrr = np.zeros(48, np.float32)
    abrr[10] = cfg["cs"]
    probe = J.calc_probe(cfg["alpha"], abrr=abrr)
    objslc = np.arange(cfg["nobj"]) % cfg["nslice_types"]
    nvar = [cfg["nvar"]] * cfg["nslice_types"]
    e = J.setup(2, nvar, objslc, [0] * cfg["nslice_types"], cfg["ndetper"], len(dets), 1)
    assert e == [0, 0, 0, 0], e
    for s, gr in enumerate(sp.gratings):
        assert J.set_phase_grating(2, s, gr) == 0
    assert J.set_propagator(2, 0, pro) == 0
    for i, (d, m) in enumerate(dets):
        assert J.set_detector(2, i, d, m) == 0
    assert J.init_core(2) == 0
    assert J.set_incident_wave(2, probe) == 0
    nc = cfg["ncell"]
    mid = (nc // 2) * A_CELL
    if cfg["nscan"] > 1:
        pos = scan_positions(cfg["nscan"], mid, mid, A_CELL)
    else:
        pos = np.array([[0.5 * sp.a, 0.5 * sp.b]], np.float32)
    return sp, probe, pro, dets, pos


def random_phase_gratings(nx: int, ny: int, a: float, b: float, ngr: int, seed: int, max_phase: float = 3.0,
                          smooth: float = 0.03) -> np.ndarray:
    """Strong-scattering random-phase gratings t = exp(i phi) [ngr, ny, nx].

    phi starts as U(0, 2 pi) per pixel (numpy PCG64, seed), is smoothed by a
    periodic Gaussian of standard deviation `smooth` nm (0.3 A), and is then
    rescaled linearly to the range [0, max_phase] rad."""
    rng = np.random.default_rng(seed)
    qx = np.fft.fftfreq(nx, d=a / nx)
    qy = np.fft.fftfreq(ny, d=b / ny)
    g = np.exp(-2.0 * (np.pi * smooth) ** 2 * (qy[:, None] ** 2 + qx[None, :] ** 2))
    out = np.empty((ngr, ny, nx), np.complex64)
    for i in range(ngr):
        phi = rng.uniform(0.0, 2.0 * np.pi, (ny, nx))
        phi = np.fft.ifft2(np.fft.fft2(phi) * g).real
        phi = (phi - phi.min()) * (max_phase / max(phi.max() - phi.min(), 1e-30))
        out[i] = np.exp(1j * phi)
    return out


# Precision sweep: single probes on strong random-phase gratings (2 slice
# types alternating, 1 grating each), 200 slices, the pixel size of the
# 3x3-cell 256^2 grid (11.715 A / 256) on every grid, 300 kV, 25 mrad,
# aberration free, probe at the cell centre; readout every 10 slices.
PRECISION_SWEEP = dict(sizes=(256, 512, 1024, 2048), nobj=200, kv=300.0, alpha=25.0, ndetper=10,
                       dets=((0.0, 10.0), (20.0, 50.0), (80.0, 200.0)), ntype=1, seed=20261205,
                       pixel=3 * A_CELL / 256, thicknesses=(10, 50, 200))


# Frozen-phonon displacement of the workloads (sigma 0.08 A per axis) as an
# isotropic B factor for the on-device grating generator's QEP model:
# B = 8 pi^2 sigma^2 [nm^2]
BISO_PHONON = 8.0 * np.pi ** 2 * 0.008 ** 2


def layer_atoms(ncell_x: int, ncell_y: int, layer: int) -> np.ndarray:
    """Atoms of one slice layer for the grating generator: [natom, 5] rows of
    fractional x, y, z, occupancy, type (0 = A, 1 = B, 2 = O)."""
    rows = [((ix + fx) / ncell_x, (iy + fy) / ncell_y, 0.0, 1.0, t)
            for iy in range(ncell_y) for ix in range(ncell_x) for (t, fx, fy) in LAYERS[layer]]
    return np.asarray(rows, np.float32)


def form_factor_tables(nx: int, ny: int, a: float, b: float, seed: int, kv: float = 300.0):
    """Radial form factors [3, nk] (complex64, nm) of the workload's three
    Gaussian atom types, sampled as CJEElaSca samples its tables (nk = 12 max(nx,
    ny), sk = max(nx / a, ny / b) / nk), scaled so that the generator's grating
    phase c V' (c = lambda / (4 pi a b)) equals sigma V(r):
        f(q) = (4 pi sigma / lambda) sum_i A_i 2 pi w_i^2 exp(-2 pi^2 w_i^2 q^2).
    Returns (ff, sk)."""
    amp, wid = atom_params(seed)
    nk = 12 * max(nx, ny)
    sk = max(nx / a, ny / b) / nk
    e0 = _ME0 * _C0 ** 2 / _QEL / 1000.0
    lam = _C0 * _HPL / _QEL * 1.0e6 / np.sqrt(kv * (kv + 2 * e0))      # nm
    k = 4.0 * np.pi * interaction_constant(kv) / lam
    q = np.arange(nk) * sk
    ff = np.zeros((3, nk), np.complex64)
    for t in range(3):
        ff[t] = k * sum(amp[t, i] * 2 * np.pi * wid[t, i] ** 2 * np.exp(-2 * np.pi ** 2 * wid[t, i] ** 2 * q * q)
                        for i in range(2))
    return ff, float(sk)
