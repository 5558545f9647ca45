"""Test infrastructure, not product code: an FP64 NumPy restatement of the RF
preparation of the reference, the checker for ``wust_dtft`` and
``waveforminversionust_b200.prepare``.  Only the tests import it.

* ``geometry``  Runtime/matlab/wust_geometry.m:1-35 (pixel-edge grid, nearest
  sample, 1-based column-major indices)
* ``dtft``      Runtime/matlab/wust_prepare.m:30-37 (per transmitter,
  kernel = exp(-2 pi i f t') dt, single(kernel * traces), inactive traces 0)
* ``prepare``   wust_prepare.m:1-68 with wust_prepare_observations.m:41-80
  (masked values zeroed, frequencies sorted, homogeneous-tof phase, norms)
"""
from __future__ import annotations

import numpy as np


def geometry(shape_yx, origin_yx, spacing_yx, tx, rx):
    y = origin_yx[0] + (np.arange(shape_yx[0]) + 0.5) * spacing_yx[0]
    x = origin_yx[1] + (np.arange(shape_yx[1]) + 0.5) * spacing_yx[1]
    out = []
    for xy in (np.asarray(tx, float), np.asarray(rx, float)):
        ix = np.array([int(np.argmin(np.abs(x - p[0]))) for p in xy])
        iy = np.array([int(np.argmin(np.abs(y - p[1]))) for p in xy])
        out.append(((iy + 1) + len(y) * ix, np.stack([x[ix], y[iy]], 1)))
    return x, y, out[0], out[1]


def dtft(time_s, freqs, pressure, active):
    """pressure [time, rx, tx] real; active [tx, rx] -> complex64 [tx, rx, f]."""
    t = np.asarray(time_s, float).ravel()
    f = np.asarray(freqs, float).ravel()
    dt = t[1] - t[0]
    kernel = np.exp(-2j * np.pi * f[:, None] * t[None, :]) * dt
    nt = pressure.shape[2]
    out = np.zeros((nt, pressure.shape[1], f.size), np.complex64)
    for k in range(nt):
        traces = np.asarray(pressure[:, :, k], float).copy()
        traces[:, ~np.asarray(active[k], bool)] = 0
        out[k] = (kernel @ traces).astype(np.complex64).T
    return out


def prepare(time_s, freqs, pressure, mask, shape_yx, origin_yx, spacing_yx, tx, rx, phase="none", c_geom=1500.0):
    f = np.asarray(freqs, float).ravel()
    mask = np.asarray(mask, bool)
    if mask.ndim == 2:
        mask = np.repeat(mask[:, :, None], f.size, axis=2)
    x, y, (ti, ts), (ri, rs) = geometry(shape_yx, origin_yx, spacing_yx, tx, rx)
    Y = dtft(time_s, f, pressure, mask.any(axis=2))
    Y[~mask] = 0
    order = np.argsort(f, kind="stable")
    Y, mask, f = Y[:, :, order], mask[:, :, order], f[order]
    if phase == "homogeneous-tof":
        def dist(a, b):
            return np.hypot(a[:, 0][:, None] - b[:, 0][None], a[:, 1][:, None] - b[:, 1][None])
        delay = (dist(ts, rs) - dist(np.asarray(tx, float), np.asarray(rx, float))) / c_geom
        Y = (Y * np.exp(-2j * np.pi * delay[:, :, None] * f[None, None, :]).astype(np.complex64)).astype(np.complex64)
    norm = np.sum(np.abs(Y.astype(np.complex128)) ** 2, axis=(0, 1))
    return dict(x_m=x, y_m=y, tx_index=ti, rx_index=ri, Y=Y, mask=mask, frequencies_hz=f, frequency_data_norm=norm,
                valid_receiver_counts=mask.sum(axis=1))
