"""RF records from a sound-speed model: Runtime/matlab/wust_simulate.m:1-87.

``wust_simulate(model, cfg)`` takes the reference's model (c_mps [ny, nx] on
the computational grid, x_m / y_m, 1-based tx_index / rx_index,
source_pressure [n_time], dt_s) and configuration (backend, pml_size,
density_kg_m3, sound_speed_ref_mps, downsample_factor, time_offset_s,
work_dir; binary_path and device_num for the native backend), checks them as
the reference does, runs every transmitter's simulation through the
library's ``wust_simulate`` (k-Wave's 2-D first-order k-space method,
batched over transmitters on the GPU) and returns a ``wust.rf`` record:
pressure [time, receiver, transmitter] float32, sample times with the offset,
the grid positions of the array and the simulation's provenance.

Both reference backends are the same physics (the test of
Runtime/tests/test_native_pipeline.m holds them to 1e-4); here
``native-batch`` marches all transmitters together and ``matlab-serial``
one transmitter at a time, on the same kernels.  ``work_dir`` is accepted
and created as in the reference (no files are written into it), and the
native backend's ``binary_path`` / ``device_num`` are accepted and unused
(the current CUDA device runs the simulation).
"""
from __future__ import annotations

import ctypes as C
import os
import time

import numpy as np

from . import _lib
from ._lib import WustError, check

_REQUIRED = ("backend", "pml_size", "density_kg_m3", "sound_speed_ref_mps", "downsample_factor", "time_offset_s",
             "work_dir")


def _invalid(msg):
    return WustError(1, msg)


def _scalar(v):
    a = np.asarray(v, np.float64)
    if a.size != 1:
        raise _invalid("Expected a scalar")
    return float(a.ravel()[0])


def wust_simulate(model: dict, cfg: dict, stream=None) -> dict:
    import torch
    for key in _REQUIRED:
        if key not in cfg:
            raise _invalid(f"Missing {key}")
    if cfg["backend"] not in ("native-batch", "matlab-serial"):
        raise _invalid("backend must be native-batch or matlab-serial")
    c = np.asarray(model["c_mps"], np.float64)
    ny, nx = c.shape
    x = np.asarray(model["x_m"], np.float64).ravel()
    y = np.asarray(model["y_m"], np.float64).ravel()
    if not (x.size == nx and y.size == ny and np.all(np.isfinite(c)) and np.all(c > 0)):
        raise _invalid("Invalid medium")
    dx, dy = float(np.mean(np.diff(x))), float(np.mean(np.diff(y)))
    if not (dx > 0 and dy > 0 and np.max(np.abs(np.diff(x) - dx)) < dx * 1e-7
            and np.max(np.abs(np.diff(y) - dy)) < dy * 1e-7):
        raise _invalid("Uniform grid required")
    dt = _scalar(model["dt_s"])
    if not (dt > 0 and c.max() * dt / min(dx, dy) <= 0.3):
        raise _invalid("CFL exceeds tested 0.3")
    rho0, c_ref = _scalar(cfg["density_kg_m3"]), _scalar(cfg["sound_speed_ref_mps"])
    if not (rho0 > 0 and c_ref >= c.max()):
        raise _invalid("Invalid density or reference speed")
    q = _scalar(cfg["downsample_factor"])
    if not (q >= 1 and q == round(q)):
        raise _invalid("Invalid decimation factor")
    pml = _scalar(cfg["pml_size"])
    if not (np.isfinite(pml) and pml >= 1 and pml == round(pml)):
        raise _invalid("Positive integer outside PML required")
    src = np.asarray(model["source_pressure"], np.float64).ravel()
    if not (src.size > 1 and np.all(np.isfinite(src))):
        raise _invalid("Finite source waveform required")
    offset = _scalar(cfg["time_offset_s"])
    if not np.isfinite(offset):
        raise _invalid("Finite source time offset required")
    tx = np.asarray(model["tx_index"], np.float64).ravel()
    rx = np.asarray(model["rx_index"], np.float64).ravel()
    for v in (tx, rx):
        if not (np.all(v == np.round(v)) and np.all(v >= 1) and np.all(v <= nx * ny) and np.unique(v).size == v.size):
            raise _invalid("Invalid/duplicate array indices")
    if cfg["backend"] == "native-batch" and tx.size < 2:
        raise _invalid("Native batch requires at least two transmitters")
    os.makedirs(str(cfg["work_dir"]), exist_ok=True)

    q, pml = int(q), int(pml)
    n_time, n_tx, n_rx = src.size, tx.size, rx.size
    ly = -(-n_time // q)
    lib = _lib.load()
    cm = np.ascontiguousarray(c.T)                    # column-major c(y, x)
    ti = np.ascontiguousarray(tx.astype(np.int32))
    ri = np.ascontiguousarray(rx.astype(np.int32))
    rf = torch.empty((n_tx, n_rx, ly), dtype=torch.float32, device="cuda")
    st = stream if stream is not None else torch.cuda.current_stream()
    batch = 0 if cfg["backend"] == "native-batch" else 1
    if "tx_batch" in cfg:
        batch = int(cfg["tx_batch"])
    t0 = time.perf_counter()
    check(lib.wust_simulate(cm.ctypes.data_as(C.c_void_p), ny, nx, dy, dx, dt, n_time, src.ctypes.data_as(C.c_void_p),
                            ti.ctypes.data_as(C.c_void_p), n_tx, ri.ctypes.data_as(C.c_void_p), n_rx, pml, c_ref,
                            rho0, q, batch, C.c_void_p(rf.data_ptr()), C.c_void_p(st.cuda_stream)))
    generation = time.perf_counter() - t0
    pressure = rf.permute(2, 1, 0).cpu().numpy()      # [time, rx, tx]
    t_array = np.arange(n_time) * dt
    saved = t_array[0] + np.arange(ly) * q * dt
    if q == 1:
        meta = dict(method="none", downsample_factor=1)
    else:
        meta = dict(method="fir-polyphase", downsample_factor=q, filter_half_length=24, kaiser_beta=8.6,
                    original_sample_rate_hz=1 / dt, saved_sample_rate_hz=1 / (q * dt), time_origin_s=float(t_array[0]),
                    nyquist_hz=1 / (2 * q * dt))
    tr, tc = (tx.astype(np.int64) - 1) % ny, (tx.astype(np.int64) - 1) // ny
    rr, rc = (rx.astype(np.int64) - 1) % ny, (rx.astype(np.int64) - 1) // ny
    return dict(schema="wust.rf", schema_version=2, data_units="Pa", measurement_provenance="self_simulated",
                pressure=pressure, time_s=saved + offset, tx_xy_m=np.stack([x[tc], y[tr]], 1),
                rx_xy_m=np.stack([x[rc], y[rr]], 1),
                simulation=dict(dt_s=dt, sound_speed_ref_mps=c_ref, generation_seconds=generation,
                                filter_seconds=0.0, resampling=meta, config=dict(cfg),
                                axis_order="time,receiver,transmitter",
                                physics="2D linear acoustics; scalar density; zero attenuation"))
