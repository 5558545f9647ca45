"""Per-frequency misfit, slowness gradient and directional curvature.

Mirrors Runtime/matlab/wust_oracle.m (``[loss, gradient, cache] =
wust_oracle(c, obs, fi, cfg)``) and Runtime/matlab/directional_curvature.m on
the GPU library: forward solve of all transmitters, receiver gather, masked
source fit a = p^H d / p^H p, residual and loss, adjoint solve, mass-stencil
adjoint and the FP64 gradient accumulation all run on the device in one C
call (``wust_solver_oracle``).  Frequencies are indexed from 0 here.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from ._lib import WustError, check
from .solver import HelmholtzSolver


@dataclass
class Observations:
    """Prepared observations (the fields of wust.measurements that the path reads,
    wust_prepare_observations.m:69-80).  Indices are 1-based column-major."""
    x_m: np.ndarray
    y_m: np.ndarray
    tx_index: np.ndarray
    rx_index: np.ndarray
    frequencies_hz: np.ndarray
    Y: np.ndarray                 # (n_tx, n_rx, n_f) complex
    mask: np.ndarray              # (n_tx, n_rx, n_f) bool
    shape_yx: tuple = field(default=None)

    def __post_init__(self):
        self.x_m = np.asarray(self.x_m, np.float64).ravel()
        self.y_m = np.asarray(self.y_m, np.float64).ravel()
        self.tx_index = np.asarray(self.tx_index, np.int64).ravel()
        self.rx_index = np.asarray(self.rx_index, np.int64).ravel()
        self.frequencies_hz = np.asarray(self.frequencies_hz, np.float64).ravel()
        self.mask = np.asarray(self.mask, bool)
        self.Y = np.where(self.mask, np.asarray(self.Y), 0)
        if self.shape_yx is None:
            self.shape_yx = (self.y_m.size, self.x_m.size)

    @property
    def n_tx(self) -> int:
        return int(self.tx_index.size)

    @property
    def n_rx(self) -> int:
        return int(self.rx_index.size)

    @property
    def valid_receiver_counts(self) -> np.ndarray:
        return self.mask.sum(axis=1)

    @property
    def frequency_data_norm(self) -> np.ndarray:
        return np.sum(np.abs(self.Y.astype(np.complex128)) ** 2, axis=(0, 1))


def default_config(**kw) -> dict:
    cfg = dict(backend="gpu", pml_m=None, pml_strength=10.0, stencil_bounds=(1400.0, 1700.0),
               wavenumber="continuum", dispersion=None, source_batch_size=256, precision="c64", refine_tol=1e-5)
    cfg.update(kw)
    return cfg


class _SolverPool:
    """One solver object per grid/configuration, refactored for each new model.

    wust_oracle.m builds a fresh HelmholtzSolver per call; reusing device
    buffers keeps the same semantics without re-allocating 2-3 GB per call.
    """

    def __init__(self):
        self._pool: dict = {}

    def get(self, c, obs: Observations, fi: int, cfg: dict) -> HelmholtzSolver:
        disp = cfg.get("dispersion") if cfg.get("wavenumber") == "kwave-ldr9" else None
        key = (obs.shape_yx, obs.x_m.tobytes(), obs.y_m.tobytes(), float(cfg["pml_m"]), float(cfg["pml_strength"]),
               tuple(map(float, cfg["stencil_bounds"])), cfg.get("precision", "c64"),
               int(min(cfg.get("source_batch_size", 256), obs.n_tx)), float(cfg.get("refine_tol", 1e-5)),
               None if not disp else (float(disp["time_step_s"]), float(disp["reference_speed_mps"])),
               cfg.get("correction_precision", "default"), int(cfg.get("max_ctas", 0)), int(cfg.get("chunk_count", 0)))
        f = float(obs.frequencies_hz[fi])
        s = self._pool.get(key)
        if s is None:
            s = HelmholtzSolver(obs.x_m, obs.y_m, c, None, f, -1, cfg["pml_strength"], cfg["pml_m"],
                                dict(backend="gpu", stencil_bounds=cfg["stencil_bounds"], dispersion=disp),
                                precision=cfg.get("precision", "c64"), max_sources=key[7], refine_tol=key[8],
                                correction_precision=key[10], max_ctas=key[11], chunk_count=key[12])
            s.generation = 0
            self._pool[key] = s
        else:
            s.refactor(c, f)
            s.generation += 1
        return s

    def clear(self):
        for s in self._pool.values():
            s.close()
        self._pool.clear()


POOL = _SolverPool()


@dataclass
class OracleState:
    """The retained state of a three-output oracle call (wust_oracle.m:81-85)."""
    solver: HelmholtzSolver
    generation: int
    rx_index: np.ndarray
    forward_rhs: int
    adjoint_rhs: int
    forward_seconds: float = 0.0
    adjoint_seconds: float = 0.0


def _host_c(a, dtype):
    return np.asfortranarray(np.asarray(a, dtype=dtype))


def wust_oracle(c, obs: Observations, fi: int, cfg: dict, nargout: int = 2, solver: HelmholtzSolver | None = None):
    """Source-projected least squares at frequency ``fi`` (0-based).

    ``nargout`` follows wust_oracle.m:5-6: 1 -> loss, 2 -> (loss, gradient),
    3 -> (loss, gradient, state for ``directional_curvature``).  A CUDA
    tensor ``c`` stays on the device and the gradient comes back as a CUDA
    float64 tensor [ny, nx]; otherwise both are host NumPy arrays.
    """
    need_gradient = nargout > 1
    retain = nargout > 2
    ny, nx = obs.shape_yx
    on_device = isinstance(c, torch.Tensor) and c.is_cuda
    if not on_device:
        c = np.asarray(c, np.float64)
    if solver is None:
        solver = POOL.get(c, obs, fi, cfg)
    lib = _lib.load()
    tx = np.ascontiguousarray(obs.tx_index, dtype=np.int32)
    rx = np.ascontiguousarray(obs.rx_index, dtype=np.int32)
    Y = _host_c(obs.Y[:, :, fi], np.complex64)
    mask = _host_c(obs.mask[:, :, fi], np.uint8)
    loss = C.c_double()
    grad = None
    if need_gradient:
        # column-major [y, x]: a contiguous [x, y] tensor on the device
        grad = torch.empty((nx, ny), dtype=torch.float64, device="cuda") if on_device else np.zeros((ny, nx), order="F")
    gptr = None if grad is None else C.c_void_p(grad.data_ptr() if on_device else grad.ctypes.data)
    flags = (_lib.NEED_GRADIENT if need_gradient else 0) | (_lib.RETAIN_STATE if retain else 0)
    bs = int(cfg.get("source_batch_size") or obs.n_tx)
    check(lib.wust_solver_oracle(C.c_void_p(solver.handle), tx.ctypes.data_as(C.c_void_p), tx.size,
                                 rx.ctypes.data_as(C.c_void_p), rx.size, Y.ctypes.data_as(C.c_void_p),
                                 mask.ctypes.data_as(C.c_void_p), bs, flags, C.byref(loss), gptr))
    if not np.isfinite(loss.value):
        raise WustError(10, "Nonfinite objective/gradient")
    if on_device and grad is not None:
        grad = grad.t()
    if nargout == 1:
        return loss.value
    if nargout == 2:
        return loss.value, grad
    state = OracleState(solver=solver, generation=getattr(solver, "generation", 0), rx_index=obs.rx_index,
                        forward_rhs=obs.n_tx, adjoint_rhs=obs.n_tx)
    return loss.value, grad, state


def directional_curvature(state: OracleState, direction, rx_index=None, receiver_mask=None) -> float:
    """Gauss-Newton curvature along ``direction`` with frozen source scales
    (directional_curvature.m:1-26); reuses the retained factors and fields."""
    s = state.solver
    if getattr(s, "generation", 0) != state.generation:
        raise WustError(1, "oracle state is stale: the solver was refactored after it was produced")
    d = np.asfortranarray(np.asarray(direction, np.float64))
    if d.shape != s.shape:
        raise WustError(1, "direction must be [ny, nx]")
    out = C.c_double()
    check(_lib.load().wust_solver_curvature(C.c_void_p(s.handle), d.ctypes.data_as(C.c_void_p), C.byref(out)))
    return out.value


def gauss_newton_product(state: OracleState, direction):
    """(Re(J^H J d), d' J^H J d): the Gauss-Newton Hessian-vector product of
    the misfit along ``direction`` with the source scales frozen (the product
    behind directional_curvature.m's quadratic form), reusing the retained
    factors and fields.  A CUDA tensor direction gives a CUDA tensor product."""
    s = state.solver
    if getattr(s, "generation", 0) != state.generation:
        raise WustError(1, "oracle state is stale: the solver was refactored after it was produced")
    if tuple(direction.shape) != s.shape:
        raise WustError(1, "direction must be [ny, nx]")
    ny, nx = s.shape
    kappa = C.c_double()
    lib = _lib.load()
    if isinstance(direction, torch.Tensor) and direction.is_cuda:
        d = direction.detach().to(torch.float64).t().contiguous()
        out = torch.empty((nx, ny), dtype=torch.float64, device="cuda")
        check(lib.wust_solver_gauss_newton_product(C.c_void_p(s.handle), C.c_void_p(d.data_ptr()),
                                                   C.c_void_p(out.data_ptr()), C.byref(kappa)))
        return out.t(), kappa.value
    d = np.asfortranarray(np.asarray(direction, np.float64))
    out = np.zeros((ny, nx), order="F")
    check(lib.wust_solver_gauss_newton_product(C.c_void_p(s.handle), d.ctypes.data_as(C.c_void_p),
                                               out.ctypes.data_as(C.c_void_p), C.byref(kappa)))
    return out, kappa.value


def gradient_device(c: torch.Tensor, obs: Observations, fi: int, cfg: dict, solver: HelmholtzSolver,
                    grad_out: torch.Tensor, tx_dev: torch.Tensor, rx_dev: torch.Tensor, Y_dev: torch.Tensor,
                    mask_dev: torch.Tensor) -> float:
    """One gradient with every array already resident in HBM (bench helper).

    ``c`` and ``grad_out`` are float64 CUDA tensors whose memory is column-
    major [y, x]; observations are CUDA tensors in the C layout of
    ``wust_solver_oracle``.
    """
    lib = _lib.load()
    check(lib.wust_solver_refactor(C.c_void_p(solver.handle), C.c_void_p(c.data_ptr()), None,
                                   C.c_double(float(obs.frequencies_hz[fi]))))
    loss = C.c_double()
    check(lib.wust_solver_oracle(C.c_void_p(solver.handle), C.c_void_p(tx_dev.data_ptr()), obs.n_tx,
                                 C.c_void_p(rx_dev.data_ptr()), obs.n_rx, C.c_void_p(Y_dev.data_ptr()),
                                 C.c_void_p(mask_dev.data_ptr()), int(cfg.get("source_batch_size") or obs.n_tx),
                                 _lib.NEED_GRADIENT, C.byref(loss), C.c_void_p(grad_out.data_ptr())))
    return loss.value
