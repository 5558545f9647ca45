"""RF preparation: real RF records -> canonical complex observations.

Mirrors Runtime/matlab/wust_prepare.m:1-68 (with the parts of
wust_prepare_observations.m:1-109 and wust_geometry.m:1-35 that it uses):
the arguments are validated on the host first, the dt-weighted DTFT of every
active trace runs on the GPU (``wust_dtft``: FP64 phases and sums, complex
single result, inactive channels zero), and the canonicalisation (snapped
geometry, ascending frequencies, masks, data norms) and the optional
homogeneous time-of-flight phase correction run on the host, as they touch
only n_tx x n_rx x n_f values.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import WustError, check

_REQUIRED = ("grid", "frequencies_hz", "c_geom_mps", "phase_correction", "mask", "data_units",
             "measurement_provenance")
_GRID = ("shape_yx", "origin_yx_m", "spacing_yx_m", "origin_kind")


def _invalid(msg):
    return WustError(1, msg)


def wust_geometry(grid: dict, tx, rx) -> dict:
    """Pixel-centre sampling coordinates and the grid samples nearest to the
    physical transmitter and receiver positions (wust_geometry.m:1-35)."""
    if sorted(grid) != sorted(_GRID):
        raise _invalid("Explicit grid fields required")
    n = np.asarray(grid["shape_yx"], np.float64).ravel()
    origin = np.asarray(grid["origin_yx_m"], np.float64).ravel()
    spacing = np.asarray(grid["spacing_yx_m"], np.float64).ravel()
    if not (n.size == 2 and np.all(np.isfinite(n) & (n >= 3) & (n == np.round(n))) and origin.size == 2
            and np.all(np.isfinite(origin)) and spacing.size == 2 and np.all(np.isfinite(spacing) & (spacing > 0))
            and grid["origin_kind"] == "pixel_edge"):
        raise _invalid("Invalid grid shape/origin/spacing")
    y = origin[0] + (np.arange(int(n[0])) + 0.5) * spacing[0]
    x = origin[1] + (np.arange(int(n[1])) + 0.5) * spacing[1]

    def snap(xy):
        xy = np.asarray(xy)
        if not (np.isrealobj(xy) and xy.ndim == 2 and xy.shape[1] == 2 and xy.shape[0] > 0
                and np.all(np.isfinite(xy))):
            raise _invalid("Positions must be finite [N,2] physical [x,y]")
        xy = xy.astype(np.float64)
        if not np.all((xy[:, 0] >= x[0]) & (xy[:, 0] <= x[-1]) & (xy[:, 1] >= y[0]) & (xy[:, 1] <= y[-1])):
            raise _invalid("Array outside grid sampling coordinates")
        ix = np.argmin(np.abs(x[:, None] - xy[None, :, 0]), axis=0)
        iy = np.argmin(np.abs(y[:, None] - xy[None, :, 1]), axis=0)
        index = (iy + 1 + y.size * ix).astype(np.int64)          # 1-based column-major
        if np.unique(index).size != index.size:
            raise _invalid("Distinct elements in one array collapse onto a grid sample")
        return index, np.stack([x[ix], y[iy]], axis=1)

    ti, ts = snap(tx)
    ri, rs = snap(rx)
    return dict(x_m=x, y_m=y, tx_index=ti, rx_index=ri, tx_xy_m=np.asarray(tx, np.float64),
                rx_xy_m=np.asarray(rx, np.float64), tx_snapped_xy_m=ts, rx_snapped_xy_m=rs)


def _pair_distance(a, b):
    return np.hypot(a[:, 0][:, None] - b[:, 0][None, :], a[:, 1][:, None] - b[:, 1][None, :])


def dtft_device(time_s, frequencies_hz, pressure, active, stream=None):
    """Y[tx, rx, k] = single(sum_t exp(-2 pi i f_k t) dt rf[t, rx, tx]) on the GPU.

    ``pressure``: real [time, rx, tx] array (float32 or float64, NumPy or
    CUDA tensor); ``active``: bool [tx, rx].  Returns a complex64 CUDA tensor
    holding Y column-major, viewed as [tx, rx, frequency].
    """
    import torch
    dev = torch.device("cuda")
    t = np.ascontiguousarray(np.asarray(time_s, np.float64).ravel())
    f = np.ascontiguousarray(np.asarray(frequencies_hz, np.float64).ravel())
    if isinstance(pressure, torch.Tensor):
        p = pressure.to(dev)
        n_time, n_rx, n_tx = p.shape
        p = p.permute(2, 1, 0).contiguous()          # memory [time, rx, tx], time fastest
    else:
        a = np.asarray(pressure)
        n_time, n_rx, n_tx = a.shape
        p = torch.as_tensor(np.ascontiguousarray(a.transpose(2, 1, 0)), device=dev)
    is_double = p.dtype == torch.float64
    if not is_double and p.dtype != torch.float32:
        p = p.to(torch.float32)
    act = torch.as_tensor(np.ascontiguousarray(np.asarray(active, bool).T).astype(np.uint8), device=dev)
    Y = torch.empty((f.size, n_rx, n_tx), dtype=torch.complex64, device=dev)
    st = stream if stream is not None else torch.cuda.current_stream()
    check(_lib.load().wust_dtft(t.ctypes.data_as(C.c_void_p), t.size, f.ctypes.data_as(C.c_void_p), f.size,
                                C.c_void_p(p.data_ptr()), int(is_double), n_rx, n_tx, C.c_void_p(act.data_ptr()),
                                C.c_void_p(Y.data_ptr()), C.c_void_p(st.cuda_stream)))
    return Y.permute(2, 1, 0)


def wust_prepare(rf: dict, cfg: dict) -> dict:
    """RF [time, rx, tx] -> canonical complex pressure with explicit grid
    (wust_prepare.m:1-68).  Returns the fields of wust.measurements."""
    if sorted(cfg) != sorted(_REQUIRED):
        raise _invalid("Missing or unsupported RF preparation fields")
    time_s = np.asarray(rf["time_s"], np.float64).ravel()
    if not (time_s.size >= 2 and np.all(np.isfinite(time_s))):
        raise _invalid("Invalid sample times")
    dt = time_s[1] - time_s[0]
    if not (dt > 0 and np.all(np.abs(np.diff(time_s) - dt) <= dt * 1e-6)):
        raise _invalid("Nonuniform time")
    f = np.asarray(cfg["frequencies_hz"], np.float64).ravel()
    if not np.all(np.isfinite(f) & (f > 0) & (f < 0.5 / dt)):
        raise _invalid("Frequency outside saved Nyquist")
    tx_xy = np.asarray(rf["tx_xy_m"])
    rx_xy = np.asarray(rf["rx_xy_m"])
    n_tx, n_rx, n_f = tx_xy.shape[0], rx_xy.shape[0], f.size
    pressure = rf["pressure"]
    shape = tuple(pressure.shape)
    real = (not pressure.is_complex()) if hasattr(pressure, "is_complex") else np.isrealobj(pressure)
    if not (real and len(shape) in (2, 3) and (shape + (1,))[:3] == (time_s.size, n_rx, n_tx)):
        raise _invalid("RF must be real [time,rx,tx] pressure")
    if len(shape) == 2:
        pressure = pressure.reshape(shape + (1,))
    m = np.asarray(cfg["mask"])
    if not np.all((m == 0) | (m == 1)):
        raise _invalid("Mask must contain 0/1")
    mask = m.astype(bool)
    if mask.shape == (n_tx, n_rx):
        mask = np.repeat(mask[:, :, None], n_f, axis=2)
    if mask.ndim == 2:
        mask = mask[:, :, None]
    if mask.shape != (n_tx, n_rx, n_f):
        raise _invalid("RF mask must be [tx,rx] or [tx,rx,frequency]")
    geo = wust_geometry(cfg["grid"], tx_xy, rx_xy)            # wust_prepare_observations.m:5
    if np.unique(f).size != f.size:
        raise _invalid("Frequencies must be finite, positive and unique")
    if cfg["data_units"] not in ("Pa*s", "instrument_units", "unknown"):
        raise _invalid("Explicit supported units and normalization required")
    phase = str(cfg["phase_correction"])
    if phase not in ("none", "homogeneous-tof"):
        raise _invalid("Unsupported phase policy")
    if phase == "homogeneous-tof":
        c_geom = cfg["c_geom_mps"]
        if not (np.isscalar(c_geom) and np.isfinite(c_geom) and c_geom > 0):
            raise _invalid("c_geom_mps must be a positive finite scalar")

    if not mask.any():
        raise _invalid("Empty observations or nonfinite pressure on a valid channel")

    Y = dtft_device(time_s, f, pressure, mask.any(axis=2)).cpu().numpy()   # wust_prepare.m:30-37
    # wust_prepare_observations.m:41-65: masked values zeroed, frequencies ascending
    Y[~mask] = 0
    order = np.argsort(f, kind="stable")
    Y, mask, f_sorted = Y[:, :, order], mask[:, :, order], f[order]
    obs = dict(geo)
    obs.update(schema="wust.measurements", schema_version=2, Y=Y, mask=mask, frequencies_hz=f_sorted,
               fourier_sign=-1, shape_yx=(geo["y_m"].size, geo["x_m"].size), n_tx=n_tx, n_rx=n_rx,
               valid_receiver_counts=mask.sum(axis=1), grid=cfg["grid"], data_units=cfg["data_units"],
               spectrum_normalization="dtft_dt", pressure_type="total_pressure")
    obs["preparation"] = dict(input_fourier_sign=-1, conversion="none", input_frequencies_hz=f,
                              canonical_to_input_permutation_1based=order + 1, input_pressure_axes="tx,rx,frequency",
                              input_mask_axes="tx,rx,frequency", phase_correction="none",
                              masked_values_policy="zero_after_preserving_mask", input_precision="single",
                              measurement_provenance=cfg["measurement_provenance"])
    if phase == "homogeneous-tof":                               # wust_prepare.m:53-60
        measured = _pair_distance(obs["tx_xy_m"], obs["rx_xy_m"])
        snapped = _pair_distance(obs["tx_snapped_xy_m"], obs["rx_snapped_xy_m"])
        delay = (snapped - measured) / float(cfg["c_geom_mps"])
        ph = np.exp(-2j * np.pi * delay[:, :, None] * f_sorted[None, None, :])
        obs["Y"] = (obs["Y"] * ph.astype(np.complex64)).astype(np.complex64)
        obs["preparation"]["geometry_reference_speed_mps"] = float(cfg["c_geom_mps"])
    obs["frequency_data_norm"] = np.sum(np.abs(obs["Y"].astype(np.complex128)) ** 2, axis=(0, 1))
    obs["preparation"].update(sampling_interval_s=dt, mask_shape=np.asarray(cfg["mask"]).shape,
                              valid_mask_elements=int(mask.sum()), phase_correction=phase)
    obs["saved_dt_s"] = dt
    if "simulation" in rf:
        obs["simulation"] = rf["simulation"]
    return obs


def to_observations(obs: dict):
    """The fields the gradient path reads, as ``objective.Observations``."""
    from .objective import Observations
    return Observations(obs["x_m"], obs["y_m"], obs["tx_index"], obs["rx_index"], obs["frequencies_hz"], obs["Y"],
                        obs["mask"])


def _axes_layout(a, axes: str):
    """[tx, rx, frequency] from a declared axis order."""
    if axes == "tx,rx,frequency":
        return a
    if axes == "frequency,tx,rx":
        return np.moveaxis(a, 0, 2)
    raise _invalid(f"Unsupported declared axes: {axes}")


def wust_prepare_observations(inp: dict) -> dict:
    """Canonical observations from a ``wust.frequency_input`` or a
    ``wust.measurements`` artifact (wust_prepare_observations.m:1-109): the
    geometry snapped to the grid (and, for canonical input, its sampling
    indices checked against that), declared units and normalisation,
    [tx, rx, frequency] layout, a 0/1 mask with masked values zeroed, the
    Fourier sign brought to -1 (conjugation only for declared real
    time-domain pressure) and ascending frequencies.  ``inp`` holds the
    artifact's metadata, its arrays and the declared ``pressure_axes`` /
    ``mask_axes`` of frequency input."""
    schema = inp.get("schema")
    if schema not in ("wust.frequency_input", "wust.measurements") or inp.get("schema_version") != 2:
        raise WustError(1, "Expected a supported WUST v2 schema")
    canonical = schema == "wust.measurements"
    geo = wust_geometry(inp["grid"], inp["tx_xy_m"], inp["rx_xy_m"])
    if canonical and not (np.array_equal(np.asarray(inp["tx_index"]).ravel().astype(np.int64), geo["tx_index"])
                          and np.array_equal(np.asarray(inp["rx_index"]).ravel().astype(np.int64), geo["rx_index"])):
        raise _invalid("Canonical sampling indices disagree with geometry")
    f = np.asarray(inp["frequencies_hz"], np.float64).ravel()
    if not (f.size and np.all(np.isfinite(f) & (f > 0)) and np.unique(f).size == f.size):
        raise _invalid("Frequencies must be finite, positive and unique")
    if inp.get("pressure_type") != "total_pressure":
        raise _invalid("Ingestion requires total complex pressure, not scattered fields or ratios")
    units, norm = inp.get("data_units"), inp.get("spectrum_normalization")
    if units not in ("Pa*s", "instrument_units", "unknown") or norm not in ("dtft_dt", "discrete_sum", "unknown"):
        raise _invalid("Explicit supported units and normalization required")
    if units == "Pa*s" and norm != "dtft_dt":
        raise _invalid("Pa*s requires the dt-weighted DTFT normalization")
    nt, nr, nf = geo["tx_index"].size, geo["rx_index"].size, f.size
    sign = inp.get("fourier_sign")
    if canonical:
        if not (np.isscalar(sign) and sign == -1 and np.all(np.diff(f) > 0)):
            raise _invalid("Canonical observations require Fourier sign -1 and strictly increasing frequencies")
        Y, mask = np.asarray(inp["Y"]), np.asarray(inp["mask"])
        p_axes = m_axes = "tx,rx,frequency"
    else:
        p_axes, m_axes = inp["pressure_axes"], inp["mask_axes"]
        Y = _axes_layout(np.asarray(inp["pressure"]), p_axes)
        mask = np.asarray(inp["mask"])
        if m_axes == "tx,rx":
            if mask.shape != (nt, nr):
                raise _invalid("Mask shape mismatch")
            mask = np.repeat(mask[:, :, None], nf, axis=2)
        else:
            mask = _axes_layout(mask, m_axes)
    if Y.ndim == 2:
        Y = Y[:, :, None]
    if mask.ndim == 2:
        mask = mask[:, :, None]
    if Y.dtype not in (np.complex64, np.complex128) or Y.shape != (nt, nr, nf):
        raise _invalid("Pressure axes/shape mismatch")
    if mask.shape != (nt, nr, nf) or not np.all((mask == 0) | (mask == 1)):
        raise _invalid("Mask must contain only booleans/0/1")
    mask = mask.astype(bool)
    if not (mask.any() and np.all(np.isfinite(Y[mask]))):
        raise _invalid("Empty observations or nonfinite pressure on a valid channel")
    Y = Y.copy()
    Y[~mask] = 0
    order = np.arange(nf)
    conversion = "none"
    if not canonical:
        if not (np.isscalar(sign) and sign in (-1, 1)):
            raise _invalid("Declare Fourier sign -1 or +1; unknown conventions are rejected")
        if sign == 1:
            if inp.get("real_pressure") is not True:
                raise _invalid("Conjugation requires declared real time-domain pressure")
            Y = np.conj(Y)
            conversion = "conjugate"
        order = np.argsort(f, kind="stable")
        Y, mask = Y[:, :, order], mask[:, :, order]
    obs = dict(geo)
    obs.update(schema="wust.measurements", schema_version=2, Y=Y, mask=mask, frequencies_hz=f[order], fourier_sign=-1,
               shape_yx=(geo["y_m"].size, geo["x_m"].size), n_tx=nt, n_rx=nr,
               valid_receiver_counts=mask.sum(axis=1),
               frequency_data_norm=np.sum(np.abs(Y.astype(np.complex128)) ** 2, axis=(0, 1)),
               grid=inp["grid"], data_units=units, spectrum_normalization=norm, pressure_type="total_pressure")
    if canonical and "preparation" in inp:
        obs["preparation"] = inp["preparation"]
    else:
        obs["preparation"] = dict(input_fourier_sign=sign, conversion=conversion, input_frequencies_hz=f,
                                  canonical_to_input_permutation_1based=order + 1, input_pressure_axes=p_axes,
                                  input_mask_axes=m_axes, phase_correction="none",
                                  masked_values_policy="zero_after_preserving_mask",
                                  input_precision="single" if Y.dtype == np.complex64 else "double",
                                  measurement_provenance=inp.get("measurement_provenance", "unknown"))
    return obs
