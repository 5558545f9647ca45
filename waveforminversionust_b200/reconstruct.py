"""Frequency-continuation NCG reconstruction, Runtime/matlab/wust_reconstruct.m:1-74.

Every schedule entry runs one oracle call (assembly + factor + forward +
adjoint on the GPU), the ROI/filter and PR/FR rules, one directional
curvature solve that reuses the same factors, the linearized step and the
slowness-space projection.  Records carry the same per-step timings.

With ``ncg_device`` (the default) the model, gradient, filtered gradient and
directions stay in device memory for the whole loop: the ROI/filter, the
direction, the slope and the projection run through the library's
``wust_ncg_*`` entry points, and only scalars (loss, curvature, slope, step)
reach the host.  ``ncg_device=False`` runs those rules in NumPy on the host,
as the reference does in MATLAB.
"""
from __future__ import annotations

import time

import ctypes as C

import numpy as np

from . import _lib
from ._lib import WustError, check
from .ncg import linearized_step_length, ncg_direction, project_slowness_update, roi_gradient
from .objective import POOL, Observations, directional_curvature, wust_oracle

_REQUIRED = ("backend", "bounds_mps", "max_update_mps", "step_damping", "source_batch_size", "pml_strength", "pml_m",
             "stencil_bounds", "wavenumber", "filter_cutoff", "filter_order", "update_mask")
_ALLOWED = _REQUIRED + ("dispersion", "frequency_schedule_hz", "max_updates", "save_history",
                        "evaluate_final_residual", "precision", "ncg_device", "correction_precision")


def _prepare(obs: Observations, initial, cfg: dict) -> dict:
    """Configuration admission (wust_reconstruct.m:124-211, the parts on the path)."""
    if not all(k in cfg for k in _REQUIRED) or not all(k in _ALLOWED for k in cfg):
        raise WustError(1, "Missing or unsupported reconstruction config fields")
    cfg = dict(cfg)
    for k in ("pml_m", "pml_strength", "max_update_mps", "step_damping", "source_batch_size", "filter_order"):
        v = cfg[k]
        if not (np.isscalar(v) and np.isfinite(v) and v > 0):
            raise WustError(1, f"Expected positive finite {k}")
    for k in ("bounds_mps", "stencil_bounds"):
        b = np.asarray(cfg[k], np.float64).ravel()
        if b.size != 2 or not np.all(np.isfinite(b)) or b[0] <= 0 or b[1] <= b[0]:
            raise WustError(1, "Invalid speed bounds")
    if cfg["backend"] != "gpu" or cfg["wavenumber"] not in ("continuum", "kwave-ldr9"):
        raise WustError(1, "Unsupported backend/wavenumber")
    initial = np.asarray(initial, np.float64)
    if initial.shape != obs.shape_yx or not np.all(np.isfinite(initial)) or np.any(
            initial < cfg["bounds_mps"][0]) or np.any(initial > cfg["bounds_mps"][1]):
        raise WustError(1, "Initial map must match grid and speed bounds")
    mask = np.asarray(cfg["update_mask"])
    if mask.shape != initial.shape or not np.all((mask == 0) | (mask == 1)):
        raise WustError(1, "Invalid update mask")
    cfg["update_mask"] = mask.astype(bool)
    full = obs.frequencies_hz if cfg.get("frequency_schedule_hz") is None else np.asarray(
        cfg["frequency_schedule_hz"], np.float64).ravel()
    schedule = []
    for f in full:
        hit = np.nonzero(obs.frequencies_hz == f)[0]
        if hit.size == 0:
            raise WustError(1, "Schedule frequencies must exactly match observations")
        schedule.append(int(hit[0]))
    cfg["planned_schedule_length"] = len(schedule)
    if cfg.get("max_updates") is not None:
        schedule = schedule[:int(cfg["max_updates"])]
    cfg["schedule"] = schedule
    cfg.setdefault("save_history", False)
    cfg.setdefault("evaluate_final_residual", False)
    evaluated = sorted(set(schedule)) if not cfg["evaluate_final_residual"] else list(range(obs.frequencies_hz.size))
    if evaluated and np.any(obs.valid_receiver_counts[:, evaluated] < 2):
        raise WustError(1, "Source-scale fitting requires two valid receivers per evaluated TX/frequency")
    ny, nx = obs.shape_yx
    interior = np.ones((ny, nx), bool)
    interior[[0, -1], :] = False
    interior[:, [0, -1]] = False
    if not np.all(interior.ravel(order="F")[obs.tx_index - 1]):
        raise WustError(1, "TX and fitted RX must sample interior (non-Dirichlet) grid points")
    return cfg


def _record(step, fi, obs, loss, alpha, beta, curvature, t_step, state_solver, lin_s, rel_update):
    absres = float(np.sqrt(2 * loss))
    norm = obs.frequency_data_norm[fi]
    rec = dict(step=step + 1, frequency_hz=float(obs.frequencies_hz[fi]), loss_before_update=loss,
               absolute_residual_before_update=absres,
               relative_residual_before_update=absres / np.sqrt(norm) if norm > 0 else float("nan"),
               relative_residual_status="available" if norm > 0 else "zero_observation_energy",
               alpha=alpha, beta=beta, curvature=curvature, wall_seconds=time.perf_counter() - t_step,
               assembly_seconds=state_solver.assembly_seconds, factor_seconds=state_solver.factor_seconds,
               linearized_seconds=lin_s, fresh_factorizations=1, forward_rhs=obs.n_tx,
               adjoint_rhs=obs.n_tx, linearized_rhs=obs.n_tx, stage_id=fi + 1, loss_model_step=step)
    rec["relative_slowness_update"] = rel_update
    return rec


def _finish(obs, cfg, c, records, history, t_all) -> dict:
    n = len(cfg["schedule"])
    reason, category = "schedule_complete", "completion"
    if n == 0:
        reason, category = "zero_updates", "budget"
    elif n < cfg["planned_schedule_length"]:
        reason, category = "caller_truncated_schedule", "budget"
    result = dict(schema="wust.reconstruction", schema_version=2, c_mps=c, records=records,
                  executed_schedule=[fi + 1 for fi in cfg["schedule"]], completed_updates=n,
                  planned_schedule_length=cfg["planned_schedule_length"],
                  completion=dict(category=category, reason=reason, converged=False), final_data_residual=None)
    if history is not None:
        result["history_mps"] = np.stack(history, axis=2)
    if cfg["evaluate_final_residual"]:
        total = sum(wust_oracle(c, obs, k, cfg, nargout=1) for k in range(obs.frequencies_hz.size))
        energy = float(np.sum(obs.frequency_data_norm))
        result["final_data_residual"] = dict(
            absolute=float(np.sqrt(2 * total)), relative=float(np.sqrt(2 * total / energy)) if energy > 0 else None,
            status="available" if energy > 0 else "zero_observation_energy",
            oracle_calls=int(obs.frequencies_hz.size), forward_rhs=obs.n_tx * int(obs.frequencies_hz.size),
            adjoint_rhs=0)
    result["wall_seconds"] = time.perf_counter() - t_all
    return result


def _reconstruct_device(obs: Observations, initial, cfg: dict) -> dict:
    """The loop of wust_reconstruct.m:20-74 with every field in device memory."""
    import torch
    lib = _lib.load()
    dev = torch.device("cuda")
    ny, nx = obs.shape_yx

    def to_dev(a, dtype):
        # (ny, nx) host array -> device tensor holding it column-major
        return torch.as_tensor(np.ascontiguousarray(np.asarray(a).T), dtype=dtype, device=dev)

    def ptr(t):
        return C.c_void_p(t.data_ptr())

    initial = np.asarray(initial, np.float64)
    c0 = float(np.mean(initial))
    c = to_dev(initial, torch.float64)
    mask = to_dev(cfg["update_mask"].astype(np.uint8), torch.uint8)
    grad, roi = torch.empty_like(c), torch.empty_like(c)
    z, prev_z, direction = torch.zeros_like(c), torch.zeros_like(c), torch.zeros_like(c)
    tx = torch.as_tensor(obs.tx_index.astype(np.int32), device=dev)
    rx = torch.as_tensor(obs.rx_index.astype(np.int32), device=dev)
    obs_dev = {}
    records = []
    history = [initial.copy()] if cfg["save_history"] else None
    prev_gz, last, solver = 0.0, None, None
    bs = int(cfg.get("source_batch_size") or obs.n_tx)
    lo, hi = map(float, cfg["bounds_mps"])
    t_all = time.perf_counter()
    for step, fi in enumerate(cfg["schedule"]):
        t_step = time.perf_counter()
        f = float(obs.frequencies_hz[fi])
        if solver is None:
            solver = POOL.get(initial, obs, fi, cfg)
        else:
            check(lib.wust_solver_refactor(C.c_void_p(solver.handle), ptr(c), None, C.c_double(f)))
            solver.generation = getattr(solver, "generation", 0) + 1
        h = C.c_void_p(solver.handle)
        if fi not in obs_dev:
            obs_dev[fi] = (torch.as_tensor(np.ascontiguousarray(obs.Y[:, :, fi].T), dtype=torch.complex64, device=dev),
                           torch.as_tensor(np.ascontiguousarray(obs.mask[:, :, fi].T).astype(np.uint8), device=dev))
        Yd, md = obs_dev[fi]
        loss = C.c_double()
        check(lib.wust_solver_oracle(h, ptr(tx), obs.n_tx, ptr(rx), obs.n_rx, ptr(Yd), ptr(md), bs,
                                     _lib.NEED_GRADIENT | _lib.RETAIN_STATE, C.byref(loss), ptr(grad)))
        if not np.isfinite(loss.value):
            raise WustError(10, "Nonfinite objective/gradient")
        check(lib.wust_ncg_roi_gradient(h, ptr(grad), ptr(mask), c0, f, float(cfg["filter_cutoff"]),
                                        float(cfg["filter_order"]), ptr(roi), ptr(z)))
        beta, gz = C.c_double(), C.c_double()
        check(lib.wust_ncg_direction(h, ptr(roi), ptr(z), ptr(prev_z), C.c_double(prev_gz), int(fi == last),
                                     ptr(direction), C.byref(beta), C.byref(gz)))
        prev_z, z = z, prev_z
        prev_gz, last = gz.value, fi
        t_lin = time.perf_counter()
        curvature = C.c_double()
        check(lib.wust_solver_curvature(h, ptr(direction), C.byref(curvature)))
        lin_s = time.perf_counter() - t_lin
        slope = C.c_double()
        check(lib.wust_ncg_dot(h, ptr(roi), ptr(direction), C.byref(slope)))
        alpha = linearized_step_length(slope.value, curvature.value)
        rel = C.c_double()
        check(lib.wust_ncg_project(h, ptr(c), ptr(direction), C.c_double(alpha), float(cfg["step_damping"]),
                                   float(cfg["max_update_mps"]), lo, hi, ptr(mask), C.byref(rel)))
        if history is not None:
            history.append(c.cpu().numpy().T.copy())
        records.append(_record(step, fi, obs, loss.value, alpha, beta.value, curvature.value, t_step, solver, lin_s,
                               rel.value))
    return _finish(obs, cfg, c.cpu().numpy().T.copy(), records, history, t_all)


def wust_reconstruct(obs: Observations, initial, cfg: dict) -> dict:
    cfg = _prepare(obs, initial, cfg)
    if cfg.get("ncg_device", True):
        return _reconstruct_device(obs, initial, cfg)
    c = np.asarray(initial, np.float64).copy()
    mask = cfg["update_mask"]
    records = []
    history = [c.copy()] if cfg["save_history"] else None
    prev_z = np.zeros_like(c)
    prev_gz = 0.0
    direction = prev_z
    last = None
    t_all = time.perf_counter()
    for step, fi in enumerate(cfg["schedule"]):
        t_step = time.perf_counter()
        loss, g, state = wust_oracle(c, obs, fi, cfg, nargout=3)
        roi, z = roi_gradient(g, mask, obs.x_m, obs.y_m, float(np.mean(initial)), obs.frequencies_hz[fi],
                              cfg["filter_cutoff"], cfg["filter_order"])
        direction, beta, gz = ncg_direction(roi, z, prev_z, prev_gz, direction, fi == last)
        prev_z, prev_gz, last = z, gz, fi
        t_lin = time.perf_counter()
        curvature = directional_curvature(state, direction, obs.rx_index, obs.mask[:, :, fi])
        lin_s = time.perf_counter() - t_lin
        slope = float(np.sum(roi * direction))
        alpha = linearized_step_length(slope, curvature)
        old_s = 1.0 / c
        c = project_slowness_update(c, direction, alpha, cfg)
        if history is not None:
            history.append(c.copy())
        rel_update = float(
            np.linalg.norm((1.0 / c)[mask] - old_s[mask]) / max(np.linalg.norm(old_s[mask]), np.finfo(float).tiny))
        records.append(_record(step, fi, obs, loss, alpha, beta, curvature, t_step, state.solver, lin_s, rel_update))
    return _finish(obs, cfg, c, records, history, t_all)
