"""FP64 restatement of the RF simulation of Runtime/matlab/wust_simulate.m
(test infrastructure: the oracle of ``waveforminversionust_b200.simulate``;
nothing of the product imports it).

wust_simulate.m runs k-Wave's 2-D first-order k-space pseudospectral solver
(the external MATLAB toolbox's kspaceFirstOrder2D, or the vendored native
binary Runtime/third_party/kspaceFirstOrder-CUDA for the batch) with linear
acoustics, a scalar density, no absorption, a Dirichlet pressure source at
one transmitter per simulation, pressure sensors at the receivers and a PML
of ``pml_size`` cells outside the grid.  The toolbox is not part of the
reference tree and MATLAB is not available here, so this file restates the
published method (Treeby & Cox, J. Biomed. Opt. 15(2) 021314, 2010) with the
constants the vendored solver uses:

- grid expanded by the PML on every side, the medium extended with its edge
  values, masks with zeros;
- k-space correction kappa = sinc(c_ref dt |k| / 2)
  (KSpaceSolver/KSpaceFirstOrderSolver.cpp:1770-1817, generateKappa);
- staggered derivatives i k exp(+-i k d / 2) on the k-Wave wavenumber vectors
  (-N/2 .. N/2-1 for even N, ifftshifted);
- PML factors exp(-dt/2 * alpha * c_ref / d * (distance / pml_size)^4),
  alpha = 2, on the grid points and the staggered points
  (KSpaceFirstOrderSolver.cpp:2202-2260, generatePml);
- one time step (computeMainLoop, :1008-1095, linear lossless kernels of
  SolverCudaKernels.cu): velocity from the pressure gradient, velocity
  divergence, split densities, Dirichlet source (rho_x = rho_y =
  s(t) / (2 c^2) at the source point, so p(source) = s(t)), p = c^2 (rho_x +
  rho_y), pressure recorded at the sensors;
- the FIR decimation of downsampleKWaveChannelData.m (MATLAB resample(x, 1,
  q, 24, 8.6): least-squares ideal low-pass of 2 * 24 * q + 1 taps, which is
  the truncated sinc, Kaiser window beta 8.6, unit DC gain, centred so the
  first output sample keeps its time).

Parity of this restatement to the toolbox is unpinned (no k-Wave output is
available here); it is pinned by physics properties in the tests.
"""
from __future__ import annotations

import numpy as np

PML_ALPHA = 2.0


def kwave_k_vector(n: int, d: float) -> np.ndarray:
    """ifftshifted wavenumbers of one axis (kWaveGrid's convention)."""
    m = np.arange(-(n // 2), n - n // 2) if n % 2 == 0 else np.arange(-(n - 1) // 2, (n - 1) // 2 + 1)
    return np.fft.ifftshift(m * (2 * np.pi / (n * d)))


def pml_profile(n: int, pml: int, d: float, dt: float, c_ref: float, staggered: bool) -> np.ndarray:
    """Multiplicative PML factors of one axis of the expanded grid."""
    out = np.ones(n)
    shift = 0.5 if staggered else 0.0
    a = -0.5 * dt * PML_ALPHA * c_ref / d
    for i in range(pml):
        out[i] = np.exp(a * ((i + shift - pml) / (-pml)) ** 4)
        out[n - pml + i] = np.exp(a * ((i + shift + 1.0) / pml) ** 4)
    return out


def decimation_filter(q: int, half_length: int = 24, beta: float = 8.6) -> np.ndarray:
    """Taps of MATLAB resample(., 1, q, half_length, beta) (p = 1)."""
    L = 2 * half_length * q + 1
    k = np.arange(L) - half_length * q
    h = np.sinc(k / q) / q
    h = h * np.kaiser(L, beta)
    return h / h.sum()


def decimate(traces: np.ndarray, q: int, half_length: int = 24, beta: float = 8.6) -> np.ndarray:
    """[..., time] -> [..., ceil(time / q)]: y[m] = sum_j h[j] x[m q + M - j],
    M = half_length * q, x zero outside the record."""
    if q == 1:
        return traces.copy()
    h = decimation_filter(q, half_length, beta)
    M = half_length * q
    n = traces.shape[-1]
    ly = -(-n // q)
    out = np.zeros(traces.shape[:-1] + (ly,))
    for m in range(ly):
        for j in range(h.size):
            t = m * q + M - j
            if 0 <= t < n:
                out[..., m] += h[j] * traces[..., t]
    return out


def simulate(c, dy: float, dx: float, dt: float, source, tx_index, rx_index, pml: int, c_ref: float,
             rho0: float) -> np.ndarray:
    """Sensor pressure [rx, tx, time] of one Dirichlet point source per
    transmitter (1-based column-major indices into c [ny, nx]); axis 0 of c
    is k-Wave's x (spacing dy), axis 1 its y (spacing dx)."""
    c = np.asarray(c, np.float64)
    ny, nx = c.shape
    s = np.asarray(source, np.float64).ravel()
    nt = s.size
    cp = np.pad(c, pml, mode="edge")
    Ny, Nx = cp.shape
    c2 = cp * cp
    k0 = kwave_k_vector(Ny, dy)[:, None]
    k1 = kwave_k_vector(Nx, dx)[None, :]
    kappa = np.sinc(c_ref * dt * np.sqrt(k0 ** 2 + k1 ** 2) / (2 * np.pi))    # np.sinc(x) = sin(pi x)/(pi x)
    d0p, d0n = 1j * k0 * np.exp(1j * k0 * dy / 2), 1j * k0 * np.exp(-1j * k0 * dy / 2)
    d1p, d1n = 1j * k1 * np.exp(1j * k1 * dx / 2), 1j * k1 * np.exp(-1j * k1 * dx / 2)
    p0, p0s = pml_profile(Ny, pml, dy, dt, c_ref, False)[:, None], pml_profile(Ny, pml, dy, dt, c_ref, True)[:, None]
    p1, p1s = pml_profile(Nx, pml, dx, dt, c_ref, False)[None, :], pml_profile(Nx, pml, dx, dt, c_ref, True)[None, :]

    def padded(index):
        iy, ix = (np.asarray(index) - 1) % ny, (np.asarray(index) - 1) // ny
        return iy + pml, ix + pml

    ry, rx_ = padded(rx_index)
    out = np.zeros((len(rx_index), len(tx_index), nt))
    for j, t_index in enumerate(tx_index):
        sy, sx = padded([t_index])
        u0 = np.zeros((Ny, Nx)); u1 = np.zeros((Ny, Nx))
        r0 = np.zeros((Ny, Nx)); r1 = np.zeros((Ny, Nx))
        p = np.zeros((Ny, Nx))
        for n in range(nt):
            P = np.fft.fft2(p) * kappa
            u0 = p0s * (p0s * u0 - dt / rho0 * np.real(np.fft.ifft2(d0p * P)))
            u1 = p1s * (p1s * u1 - dt / rho0 * np.real(np.fft.ifft2(d1p * P)))
            du0 = np.real(np.fft.ifft2(d0n * kappa * np.fft.fft2(u0)))
            du1 = np.real(np.fft.ifft2(d1n * kappa * np.fft.fft2(u1)))
            r0 = p0 * (p0 * r0 - dt * rho0 * du0)
            r1 = p1 * (p1 * r1 - dt * rho0 * du1)
            r0[sy, sx] = r1[sy, sx] = s[n] / (2 * c2[sy, sx])
            p = c2 * (r0 + r1)
            out[:, j, n] = p[ry, rx_]
    return out
