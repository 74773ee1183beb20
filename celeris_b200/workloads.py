"""Seeded synthetic inputs with the shapes of the far-field and RCWA workloads.

No dataset is involved: every array is generated from numpy's default_rng with
the seed recorded by the caller.

Far-field metalens aperture (the psfbench geometry, cli/bench.cpp:122-135):
  square lattice of `lattice` x `lattice` sites at `period` microns, sites at
  x = (ix - (lattice-1)/2) * period (focal.cpp:47-48 centering), kept when
  r <= radius; hyperbolic focusing phase phi = -(2 pi/lambda)(sqrt(r^2+f^2)-f)
  wrapped to [0, 2 pi); |t| ~ U[0.85, 1.0]; t = |t| exp(i phi).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class Aperture:
    px: np.ndarray  # float64 [npil]
    py: np.ndarray  # float64 [npil]
    t: np.ndarray   # complex128 [npil]
    wavelength_um: float
    focal_um: float
    seed: int

    @property
    def npil(self) -> int:
        return int(self.px.shape[0])

    @property
    def k(self) -> float:
        return 2.0 * np.pi / self.wavelength_um


@dataclass
class FocalGrid:
    n: int
    half_window_um: float
    z_um: float
    cx: float = 0.0
    cy: float = 0.0

    @property
    def npix(self) -> int:
        return self.n * self.n


def metalens_aperture(lattice: int, period_um: float, radius_um: float, wavelength_um: float,
                      focal_um: float, seed: int = 0) -> Aperture:
    c = (lattice - 1) / 2.0
    iy, ix = np.meshgrid(np.arange(lattice), np.arange(lattice), indexing="ij")
    x = (ix - c) * period_um
    y = (iy - c) * period_um
    r = np.sqrt(x * x + y * y)
    keep = r <= radius_um
    x, y, r = x[keep], y[keep], r[keep]  # row-major (iy outer, ix inner) like the reference loops
    phi = -(2.0 * np.pi / wavelength_um) * (np.sqrt(r * r + focal_um * focal_um) - focal_um)
    phi = np.mod(phi, 2.0 * np.pi)
    rng = np.random.default_rng(seed)
    amp = rng.uniform(0.85, 1.0, size=x.shape[0])
    t = amp * np.exp(1j * phi)
    return Aperture(np.ascontiguousarray(x), np.ascontiguousarray(y), np.ascontiguousarray(t),
                    wavelength_um, focal_um, seed)


def metalens_70k(seed: int = 0):
    """300 x 300 sites at 0.4 um inside r <= 60 um (70,688 pillars), lambda 633 nm,
    f = 100 um; focal grid 161 x 161 over +/-5 um at z = f."""
    ap = metalens_aperture(300, 0.4, 60.0, 0.633, 100.0, seed)
    return ap, FocalGrid(161, 5.0, 100.0)


def metalens_785k(seed: int = 0):
    """1000 x 1000 sites at 0.35 um inside r <= 175 um (785,456 pillars), lambda
    532 nm, f = 1 mm; focal grid 1024 x 1024 over +/-20 um at z = f."""
    ap = metalens_aperture(1000, 0.35, 175.0, 0.532, 1000.0, seed)
    return ap, FocalGrid(1024, 20.0, 1000.0)


def rcwa_library_64():
    """Library sweep: square pillar n = 2.0 on n = 1.46 in air, period 400 nm,
    height 600 nm, 64 widths uniformly 80-360 nm (fill = w / p), M = 3
    (7 x 7 = 49 harmonics, 2N = 98), lambda 633 nm, normal incidence."""
    w = np.linspace(0.080, 0.360, 64)
    return [dict(period_um=0.4, wavelength_um=0.633, n_inc=1.0, n_sub=1.46, eps_pillar=4.0, eps_bg=1.0,
                 fill_x=float(x / 0.4), thickness_um=0.6, Mx=3) for x in w]


SHAPES = ("square", "circle", "ring")


def rcwa_uneven_4096(ncell: int = 4096, seed: int = 0, grid: int = 256):
    """Uneven batch: shape uniform in {square, circle, ring (inner/outer 0.5)}
    rasterised on a grid x grid permittivity raster (Laurent rule, squares
    included), pillar index U[1.9, 2.6], fill U[0.15, 0.85], height
    U[0.4, 0.9] um, lambda U[0.45, 0.70] um, M uniform in {3..7} ((2M+1)^2 =
    49..225 harmonics, 2N = 98..450); substrate n = 1.46, air above and around,
    period 400 nm."""
    rng = np.random.default_rng(seed)
    shape = rng.integers(0, 3, ncell)
    npil = rng.uniform(1.9, 2.6, ncell)
    fill = rng.uniform(0.15, 0.85, ncell)
    h = rng.uniform(0.4, 0.9, ncell)
    wl = rng.uniform(0.45, 0.70, ncell)
    M = rng.integers(3, 8, ncell)
    shape_code = {0: 0, 1: 1, 2: 3}  # celeris_b200.capi SHAPE_RECT / ELLIPSE / RING
    cells = []
    for i in range(ncell):
        cells.append(dict(period_um=0.4, wavelength_um=float(wl[i]), n_inc=1.0, n_sub=1.46,
                          eps_pillar=float(npil[i]) ** 2, eps_bg=1.0, fill_x=float(fill[i]),
                          thickness_um=float(h[i]), Mx=int(M[i]), shape=shape_code[int(shape[i])],
                          shape_param=0.5, grid=grid, force_laurent=1, name=SHAPES[int(shape[i])]))
    return cells


def small_aperture(npil: int = 257, seed: int = 1, spread_um: float = 8.0, wavelength_um: float = 0.55,
                   focal_um: float = 30.0):
    """Random pillars (ragged count) for quick parity checks."""
    rng = np.random.default_rng(seed)
    x = rng.uniform(-spread_um, spread_um, npil)
    y = rng.uniform(-spread_um, spread_um, npil)
    t = rng.uniform(0.5, 1.0, npil) * np.exp(1j * rng.uniform(0, 2 * np.pi, npil))
    return Aperture(x, y, t, wavelength_um, focal_um, seed)
