"""Seeded synthetic workloads with the shapes of the benchmark configurations.

No public dataset is involved: phantoms, ring arrays and masks are generated
from a seed.  Geometry follows Runtime/matlab/wust_geometry.m (pixel-edge
grid origin, centres at origin + (i + 1/2) * spacing, nearest-sample snapping
with ties to the first index, 1-based column-major indices).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from ._lib import WustError


@dataclass
class Problem:
    name: str
    x_m: np.ndarray
    y_m: np.ndarray
    dx: float
    pml_cells: int
    tx_index: np.ndarray       # 1-based
    rx_index: np.ndarray       # 1-based
    frequencies_hz: np.ndarray
    c_true: np.ndarray
    c_init: np.ndarray
    update_mask: np.ndarray

    @property
    def shape(self):
        return (self.y_m.size, self.x_m.size)

    @property
    def pml_m(self):
        return self.pml_cells * self.dx


def grid_centres(n: int, dx: float):
    origin = -n * dx / 2
    return origin + (np.arange(n) + 0.5) * dx


def snap(xy: np.ndarray, x: np.ndarray, y: np.ndarray) -> np.ndarray:
    """Nearest grid sample, first index on ties; rejects collapsed elements."""
    ix = np.argmin(np.abs(x[:, None] - xy[None, :, 0]), axis=0)
    iy = np.argmin(np.abs(y[:, None] - xy[None, :, 1]), axis=0)
    idx = (iy + 1) + y.size * ix
    if np.unique(idx).size != idx.size:
        raise WustError(1, "Distinct elements in one array collapse onto a grid sample")
    return idx.astype(np.int64)


def ring(n_elem: int, radius: float) -> np.ndarray:
    th = 2 * np.pi * np.arange(n_elem) / n_elem
    return np.stack([radius * np.cos(th), radius * np.sin(th)], axis=1)


def _smooth_noise(rng, shape, sigma_cells: float) -> np.ndarray:
    n = rng.standard_normal(shape)
    ky = np.fft.fftfreq(shape[0])[:, None]
    kx = np.fft.fftfreq(shape[1])[None, :]
    filt = np.exp(-2 * (np.pi * sigma_cells) ** 2 * (kx ** 2 + ky ** 2))
    out = np.real(np.fft.ifft2(np.fft.fft2(n) * filt))
    return out / max(out.std(), 1e-30)


def _problem(name, interior, pml, dx, n_elem, radius, n_tx, freqs, c_true, mask_radius, rng=None):
    n = interior + 2 * pml
    x = grid_centres(n, dx)
    y = grid_centres(n, dx)
    elems = ring(n_elem, radius)
    rx = snap(elems, x, y)
    step = n_elem // n_tx
    tx = rx[::step][:n_tx].copy()
    X, Y = np.meshgrid(x, y)
    mask = (X ** 2 + Y ** 2) < mask_radius ** 2
    return Problem(name=name, x_m=x, y_m=y, dx=dx, pml_cells=pml, tx_index=tx, rx_index=rx,
                   frequencies_hz=np.asarray(freqs, np.float64), c_true=c_true(X, Y),
                   c_init=np.full((n, n), 1500.0), update_mask=mask)


def config1(seed: int = 0, freqs=None) -> Problem:
    """192^2 + 16-cell PML, dx 0.4 mm, 0.5 MHz, 128-element ring r = 35 mm, 32 TX,
    three seeded elliptical inclusions (semi-axes 3-10 mm, 1450-1600 m/s).
    ``freqs`` replaces the single 0.5 MHz (the precision study runs config 1's
    geometry at twelve frequencies from 0.3 to 1.2 MHz)."""
    rng = np.random.default_rng(seed)

    def c_true(X, Y):
        c = np.full(X.shape, 1500.0)
        for _ in range(3):
            cx, cy = rng.uniform(-15e-3, 15e-3, 2)
            a, b = rng.uniform(3e-3, 10e-3, 2)
            th = rng.uniform(0, np.pi)
            xr = (X - cx) * np.cos(th) + (Y - cy) * np.sin(th)
            yr = -(X - cx) * np.sin(th) + (Y - cy) * np.cos(th)
            c[(xr / a) ** 2 + (yr / b) ** 2 < 1] = rng.uniform(1450, 1600)
        return c

    return _problem("config1", 192, 16, 0.4e-3, 128, 35e-3, 32, [0.5e6] if freqs is None else list(freqs), c_true,
                    30e-3)


def config2(seed: int = 0, freqs=None) -> Problem:
    """512^2 + 20-cell PML, dx 0.25 mm, 256-element ring r = 55 mm, all 256 TX;
    breast-like phantom (1500 m/s water, 45 mm-radius disk at 1470 m/s, 5-15
    inclusions at 1520-1580 m/s, 5 m/s Gaussian texture)."""
    rng = np.random.default_rng(seed)
    if freqs is None:
        freqs = np.linspace(0.3e6, 1.2e6, 12)

    def c_true(X, Y):
        R = np.sqrt(X ** 2 + Y ** 2)
        c = np.full(X.shape, 1500.0)
        disk = R < 45e-3
        c[disk] = 1470.0
        for _ in range(int(rng.integers(5, 16))):
            r0 = rng.uniform(0, 35e-3)
            th = rng.uniform(0, 2 * np.pi)
            rad = rng.uniform(2e-3, 8e-3)
            c[((X - r0 * np.cos(th)) ** 2 + (Y - r0 * np.sin(th)) ** 2) < rad ** 2] = rng.uniform(1520, 1580)
        c[disk] += 5.0 * _smooth_noise(rng, X.shape, 2.0)[disk]
        return c

    return _problem("config2", 512, 20, 0.25e-3, 256, 55e-3, 256, freqs, c_true, 50e-3)


def config4(seed: int = 0) -> Problem:
    """256^2 + 16-cell PML, dx 0.3 mm, 128-element ring r = 36 mm, 64 TX, 0.4/0.8 MHz."""
    rng = np.random.default_rng(seed)

    def c_true(X, Y):
        return 1500.0 + 30.0 * _smooth_noise(rng, X.shape, 8.0)

    return _problem("config4", 256, 16, 0.3e-3, 128, 36e-3, 64, [0.4e6, 0.8e6], c_true, 33e-3)


def small(seed: int = 0, n_interior: int = 48, pml: int = 8, dx: float = 0.5e-3, n_elem: int = 24,
          n_tx: int = 6, freqs=(0.3e6,)) -> Problem:
    """A seconds-scale case for parity tests against the FP64 oracle."""
    rng = np.random.default_rng(seed)
    n = n_interior + 2 * pml
    radius = 0.38 * n_interior * dx

    def c_true(X, Y):
        c = 1500.0 + 25.0 * np.exp(-((X - 2e-3) ** 2 + (Y + 1e-3) ** 2) / (2 * (0.15 * n * dx) ** 2))
        return c + 3.0 * _smooth_noise(rng, X.shape, 1.5)

    return _problem("small", n_interior, pml, dx, n_elem, radius, n_tx, list(freqs), c_true, 0.3 * n_interior * dx)
