"""Scalar rules of the NCG update, FP64 on the host (the reference keeps them on
the host as well; they touch one Ny x Nx field per step).

* ``ncg_direction``             Runtime/matlab/wust_ncg_direction.m:1-17
* ``linearized_step_length``    Runtime/matlab/linearized_step_length.m:1-11
* ``roi_gradient``              Runtime/matlab/wust_roi_gradient.m:1-10
* ``project_slowness_update``   Runtime/matlab/wust_project_slowness_update.m:1-10
* ``ringing_removal_filt``      Runtime/solver/ringingRemovalFilt.m:1-45
"""
from __future__ import annotations

import numpy as np

from ._lib import WustError


def ncg_direction(g, z, prev_z, prev_gz, previous_direction, same_frequency):
    """Clipped, preconditioned PR/FR direction with restart on non-descent."""
    g = np.asarray(g, np.float64)
    z = np.asarray(z, np.float64)
    gz = float(np.dot(g.ravel(), z.ravel()))
    beta = 0.0
    if same_frequency and prev_gz > 0:
        beta_fr = gz / prev_gz
        beta_pr = float(np.dot(g.ravel(), (z - np.asarray(prev_z, np.float64)).ravel())) / prev_gz
        beta = min(max(beta_pr, 0.0), beta_fr)
    direction = -z + beta * np.asarray(previous_direction, np.float64)
    if float(np.dot(g.ravel(), direction.ravel())) >= 0:
        direction = -z
        beta = 0.0
    if not (np.all(np.isfinite(direction)) and np.isfinite(gz) and gz >= 0):
        raise WustError(10, "Invalid preconditioned gradient")
    return direction, beta, gz


def linearized_step_length(slope: float, curvature: float) -> float:
    """Minimizer of the frozen-source quadratic along a descent direction."""
    if not (np.isfinite(slope) and np.isfinite(curvature) and curvature >= 0):
        raise WustError(10, "Nonfinite slope/curvature")
    if not (curvature > 0 or slope == 0):
        raise WustError(10, "Zero curvature with nonzero directional slope")
    return max(0.0, -slope / curvature) if curvature > 0 else 0.0


def ringing_removal_filt(xin, yin, img, c0, f, cutoff, order):
    """Radial Butterworth low-pass in k-space; cutoff 0 returns the input."""
    if not (np.isscalar(cutoff) and np.isfinite(cutoff) and cutoff >= 0):
        raise WustError(1, "cutoff must be a finite nonnegative scalar")
    if cutoff == 0:
        return img
    xin = np.asarray(xin, np.float64).ravel()
    yin = np.asarray(yin, np.float64).ravel()
    nx, ny = xin.size, yin.size
    dx = float(np.mean(np.diff(xin)))
    dy = float(np.mean(np.diff(yin)))
    kx = np.fft.fftshift((np.arange(nx) / nx) / dx)
    kx = np.where(kx >= 1 / (2 * dx), kx - 1 / dx, kx)
    ky = np.fft.fftshift((np.arange(ny) / ny) / dy)
    ky = np.where(ky >= 1 / (2 * dy), ky - 1 / dy, ky)
    KX, KY = np.meshgrid(kx, ky)
    kc = (2 * f / c0) * cutoff
    filt = 1.0 / (1.0 + ((KX ** 2 + KY ** 2) / kc ** 2) ** order)
    spec = np.fft.fftshift(np.fft.fft2(img))
    return np.real(np.fft.ifft2(np.fft.ifftshift(filt * spec)))


def roi_gradient(g, mask, x_m, y_m, c0, frequency_hz, cutoff, order):
    """M F M g: restrict before filtering so exterior gradient cannot leak in."""
    mask = np.asarray(mask, bool)
    roi = np.where(mask, g, 0.0)
    z = roi
    if cutoff > 0:
        z = ringing_removal_filt(x_m, y_m, z, c0, frequency_hz, cutoff, order)
    z = np.where(mask, z, 0.0)
    return roi, z


def project_slowness_update(c, direction, alpha, cfg):
    """Clip in slowness, then invert; outside the update mask c is unchanged."""
    c = np.asarray(c, np.float64)
    c_lo = np.maximum(c - cfg["max_update_mps"], cfg["bounds_mps"][0])
    c_hi = np.minimum(c + cfg["max_update_mps"], cfg["bounds_mps"][1])
    trial = 1.0 / c + cfg["step_damping"] * alpha * np.asarray(direction, np.float64)
    if not np.all(np.isfinite(trial)):
        raise WustError(10, "Nonfinite slowness trial")
    s_new = np.maximum(1.0 / c_hi, np.minimum(1.0 / c_lo, trial))
    return np.where(np.asarray(cfg["update_mask"], bool), 1.0 / s_new, c)
