"""HelmholtzSolver with the reference's constructor and methods, on libwust_b200.

Mirrors Runtime/solver/HelmholtzSolver.m:

* ``HelmholtzSolver(x, y, vel, atten, f, signConvention, a0, L_PML, options)``
  (:32-172) -- assembles the nine-point PML operator and factorizes it on the
  GPU; ``options`` needs ``backend`` and ``stencil_bounds`` (:34-40).
* ``solve(src, adjoint)`` (:174-203) -> wavefield, optionally virtual sources.
* ``massApply(v, adjoint)`` (:205-220).
* properties ``assembly_seconds``, ``factor_seconds``, ``massD``, ``massE``,
  ``virtualSourceMultiplier`` and the factor blocks ``Ld ... Uu``, ``invT``.

Arrays follow MATLAB layout: a field is indexed ``[y, x]`` and a stack
``[y, x, source]`` with y fastest in memory.  Inputs may be NumPy arrays
(host) or CUDA torch tensors; outputs are CUDA torch tensors of shape
``(Ny, Nx, S)`` whose memory is column-major (a permuted view of a
contiguous ``(S, Nx, Ny)`` tensor).  Only the ``gpu`` backend exists here.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import WustError, check


class _DeviceView:
    """Non-owning CUDA array view used to wrap solver-owned device blocks."""

    def __init__(self, ptr: int, shape, typestr: str, owner):
        self.__cuda_array_interface__ = {
            "shape": tuple(shape), "typestr": typestr, "data": (ptr, False), "version": 3,
            "strides": None,
        }
        self._owner = owner


def _fortran_device(a, dtype: torch.dtype) -> torch.Tensor:
    """A CUDA tensor of shape (S, Nx, Ny) contiguous == column-major (Ny, Nx, S)."""
    if isinstance(a, torch.Tensor):
        t = a.to(device="cuda", dtype=dtype)
    else:
        t = torch.as_tensor(np.asarray(a), device="cuda").to(dtype)
    if t.dim() == 2:
        t = t.unsqueeze(-1)
    if t.dim() != 3:
        raise WustError(1, "Expected a [ny,nx] or [ny,nx,n] array")
    return t.permute(2, 1, 0).contiguous()


def _medium_pointer(vel):
    """A [ny, nx] medium as a column-major float64 buffer the library reads:
    CUDA tensors stay on the device, anything else becomes a host array.
    Returns (pointer, owner to keep alive during the call)."""
    if isinstance(vel, torch.Tensor) and vel.is_cuda:
        t = vel.detach().to(torch.float64).t().contiguous()       # memory [x][y] == column-major [y, x]
        return C.c_void_p(t.data_ptr()), t
    a = np.asfortranarray(np.asarray(vel.detach().cpu().numpy() if isinstance(vel, torch.Tensor) else vel,
                                     dtype=np.float64))
    return a.ctypes.data_as(C.c_void_p), a


def _grid_vector(v) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(v, dtype=np.float64).ravel())


class HelmholtzSolver:
    """Nine-point Helmholtz/PML solver on one B200 (gpu backend of HelmholtzSolver.m)."""

    def __init__(self, x, y, vel, atten, f, signConvention, a0, L_PML, options, *,
                 precision: str = "c64", refine_tol: float = 1e-5, refine_max_iters: int = 8,
                 max_sources: int | None = None, stream: torch.cuda.Stream | None = None,
                 factor_method: str = "default", sweep_method: str = "default",
                 correction_precision: str = "default", max_ctas: int = 0, chunk_count: int = 0):
        if not isinstance(options, dict) or "backend" not in options or "stencil_bounds" not in options:
            raise WustError(1, "Explicit backend and fixed stencil_bounds are required")
        bounds = options["stencil_bounds"]
        b = np.asarray(bounds, dtype=np.float64).ravel() if bounds is not None else np.zeros(0)
        if b.size != 2 or not np.all(np.isfinite(b)) or b[0] <= 0 or b[1] <= b[0]:
            raise WustError(1, "stencil_bounds must be a positive ordered [min,max] pair")
        backend = str(options["backend"])
        if backend not in ("cpu", "gpu"):
            raise WustError(1, "backend must be cpu or gpu")
        if backend != "gpu":
            raise WustError(1, "this library implements the gpu backend only (no CPU fallback)")
        self.backend = "gpu"
        self._lib = _lib.load()
        self._x = _grid_vector(x)
        self._y = _grid_vector(y)
        ny, nx = self._y.size, self._x.size
        if tuple(vel.shape) != (ny, nx) or min(ny, nx) < 3:
            raise WustError(1, "Expected a positive finite [ny,nx] medium")
        self.shape = (ny, nx)
        disp = options.get("dispersion") or None
        opts = _lib.SolverOptions()
        opts.ny, opts.nx = ny, nx
        opts.x_m = self._x.ctypes.data_as(C.POINTER(C.c_double))
        opts.y_m = self._y.ctypes.data_as(C.POINTER(C.c_double))
        opts.frequency_hz = float(f)
        opts.sign_convention = float(signConvention)
        opts.pml_strength = float(a0)
        opts.pml_m = float(L_PML)
        opts.stencil_vmin, opts.stencil_vmax = float(b[0]), float(b[1])
        opts.dispersion = 1 if disp else 0
        if disp:
            opts.time_step_s = float(disp["time_step_s"])
            opts.reference_speed_mps = float(disp["reference_speed_mps"])
        opts.precision = _lib.PRECISION[precision]
        opts.refine_max_iters = int(refine_max_iters)
        opts.refine_tol = float(refine_tol)
        methods = {"default": 0, "gauss-jordan": 1}
        if factor_method not in methods:
            raise WustError(1, f"factor_method must be one of {sorted(methods)}")
        opts.factor_method = methods[factor_method]
        sweeps = {"default": 0, "sequential": 1}
        if sweep_method not in sweeps:
            raise WustError(1, f"sweep_method must be one of {sorted(sweeps)}")
        opts.sweep_method = sweeps[sweep_method]
        corrections = {"default": 0, "same": 1}
        if correction_precision not in corrections:
            raise WustError(1, f"correction_precision must be one of {sorted(corrections)}")
        opts.correction_precision = corrections[correction_precision]
        opts.max_sources = int(max_sources or 256)
        opts.max_ctas = int(max_ctas)
        opts.chunk_count = int(chunk_count)
        self._opts = opts
        self.precision = precision
        self.max_sources = opts.max_sources
        self._stream = stream or torch.cuda.current_stream()
        handle = C.c_void_p()
        vel_p, self._vel_keep = _medium_pointer(vel)
        att_c = None if atten is None else np.asfortranarray(np.asarray(atten, dtype=np.float64))
        if att_c is not None and not np.any(att_c):
            att_c = None
        check(self._lib.wust_solver_create(C.byref(handle), C.byref(opts), vel_p,
                                           None if att_c is None else att_c.ctypes.data_as(C.c_void_p),
                                           C.c_void_p(self._stream.cuda_stream)))
        self._h = handle
        self._read_meta()

    # -- lifecycle --------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.wust_solver_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def refactor(self, vel, f=None, atten=None):
        """Re-assemble and re-factorize for a new medium/frequency (same grid).
        A CUDA tensor medium stays on the device (no host copy)."""
        if tuple(vel.shape) != self.shape:
            raise WustError(1, "Expected a positive finite [ny,nx] medium")
        vel_p, keep = _medium_pointer(vel)
        att_c = None if atten is None else np.asfortranarray(np.asarray(atten, dtype=np.float64))
        f = self.frequency_hz if f is None else float(f)
        check(self._lib.wust_solver_refactor(self._h, vel_p,
                                             None if att_c is None else att_c.ctypes.data_as(C.c_void_p),
                                             C.c_double(f)))
        if isinstance(keep, torch.Tensor):
            keep.record_stream(self._stream)      # the library copies it on the solver stream
        self._opts.frequency_hz = f
        self._read_meta()

    def _read_meta(self):
        a, fct = C.c_double(), C.c_double()
        check(self._lib.wust_solver_timings(self._h, C.byref(a), C.byref(fct)))
        self.assembly_seconds = a.value * 1e-3
        self.factor_seconds = fct.value * 1e-3
        b, d, e = C.c_double(), C.c_double(), C.c_double()
        check(self._lib.wust_solver_stencil(self._h, C.byref(b), C.byref(d), C.byref(e)))
        self.massB, self.massD, self.massE = b.value, d.value, e.value

    @property
    def frequency_hz(self) -> float:
        return self._opts.frequency_hz

    @property
    def handle(self) -> int:
        return self._h.value

    # -- factor blocks as device views (HelmholtzSolver.m:18-24) -----------
    def block(self, name: str) -> torch.Tensor:
        ptr, r, c, p = C.c_void_p(), C.c_int(), C.c_int(), C.c_int()
        check(self._lib.wust_solver_block(self._h, name.encode(), C.byref(ptr), C.byref(r), C.byref(c), C.byref(p)))
        typestr = "<c16" if name == "mult" else "<c8"
        shape = (p.value, c.value, r.value)      # column-major pages
        t = torch.as_tensor(_DeviceView(ptr.value, shape, typestr, self), device="cuda")
        t = t.permute(2, 1, 0)
        return t if p.value > 1 else t[:, :, 0]

    def __getattr__(self, name):
        if name in ("Ld", "Ll", "Lu", "Ud", "Ul", "Uu", "Dd", "Dl", "Du", "invT"):
            return self.block(name)
        if name == "virtualSourceMultiplier":
            return self.block("mult")
        raise AttributeError(name)

    # -- solves -------------------------------------------------------------
    def solve(self, src, adjoint: bool = False, want_virtual: bool = False):
        """wvfield = H \\ src (or H' \\ src); with ``want_virtual`` also mult .* wvfield."""
        t = _fortran_device(src, torch.complex64)
        S = t.shape[0]
        if t.shape[1:] != (self.shape[1], self.shape[0]):
            raise WustError(1, "source must be [ny, nx, n]")
        outs = []
        virts = []
        for first in range(0, S, self.max_sources):
            part = t[first:first + self.max_sources]
            nb = part.shape[0]
            out = torch.empty_like(part)
            virt = torch.empty_like(part) if want_virtual else None
            check(self._lib.wust_solver_solve(self._h, C.c_void_p(part.data_ptr()), nb, int(bool(adjoint)),
                                              C.c_void_p(out.data_ptr()),
                                              None if virt is None else C.c_void_p(virt.data_ptr())))
            outs.append(out)
            if want_virtual:
                virts.append(virt)
        u = torch.cat(outs).permute(2, 1, 0) if len(outs) > 1 else outs[0].permute(2, 1, 0)
        if want_virtual:
            v = torch.cat(virts).permute(2, 1, 0) if len(virts) > 1 else virts[0].permute(2, 1, 0)
            return u, v
        return u

    def massApply(self, v, adjoint: bool):
        t = _fortran_device(v, torch.complex64)
        out = torch.empty_like(t)
        check(self._lib.wust_solver_mass_apply(self._h, C.c_void_p(t.data_ptr()), t.shape[0], int(bool(adjoint)),
                                               C.c_void_p(out.data_ptr())))
        return out.permute(2, 1, 0)

    mass_apply = massApply

    def stats(self):
        it, res, err, nl = C.c_int(), C.c_double(), C.c_double(), C.c_longlong()
        check(self._lib.wust_solver_stats(self._h, C.byref(it), C.byref(res), C.byref(err), C.byref(nl)))
        return {"refine_iters": it.value, "final_residual": res.value, "error_estimate": err.value,
                "kernel_launches": nl.value}

    def sweep_times(self):
        """Total device milliseconds and count of the sweep pairs run so far."""
        ms, n = C.c_double(), C.c_longlong()
        check(self._lib.wust_solver_sweep_times(self._h, C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def factor_stats(self):
        """How the last factorization inverted its Schur pages."""
        out = (C.c_longlong * 4)()
        check(self._lib.wust_solver_factor_stats(self._h, out))
        return {"gemms": out[0], "updates": out[1], "newton_schulz_pages": out[2], "gauss_jordan_pages": out[3]}

    def factor_info(self):
        """K split of the Newton-Schulz GEMM tiles and whether the last
        factorization ran them as thread-block clusters (1), as separate CTAs
        (0) or not at all (-1)."""
        ks, cl = C.c_int(), C.c_int()
        check(self._lib.wust_solver_factor_info(self._h, C.byref(ks), C.byref(cl)))
        return {"k_slices": ks.value, "cluster": cl.value}


def decompBlockLU(Ld, Ll, Lu, Dd, Dl, Du, Ud, Ul, Uu, stream=None, timings=False):
    """Drop-in for the decompBlockLU MEX (decompBlockLU.cu:173-396) on CUDA tensors.

    Blocks are (rows, cols) complex64 CUDA tensors in MATLAB layout (column-
    major memory, as produced by ``_fortran_device``-style permuted views or
    by passing ``t.T.contiguous().T``).  Returns invT (Ny, Ny, Nx).
    """
    lib = _lib.load()
    blocks = [_colmajor2d(b) for b in (Ld, Ll, Lu, Dd, Dl, Du, Ud, Ul, Uu)]
    Ny, Nx = Dd.shape[0], Dd.shape[1]
    invT = torch.empty((Nx, Ny, Ny), dtype=torch.complex64, device="cuda")
    ms = C.c_float()
    st = stream or torch.cuda.current_stream()
    check(lib.wust_decomp_block_lu(*[C.c_void_p(b.data_ptr()) for b in blocks], Ny, Nx, C.c_void_p(invT.data_ptr()),
                                   C.byref(ms) if timings else None, C.c_void_p(st.cuda_stream)))
    out = invT.permute(2, 1, 0)
    if timings:
        return out, {"total_gpu_ms": ms.value, "block_count": Nx}
    return out


def applyBlockLU(SRC, Ld, Ll, Lu, Ud, Ul, Uu, invT, adjoint, stream=None):
    """Drop-in for the applyBlockLU MEX (applyBlockLU.cu:291-481) on CUDA tensors."""
    lib = _lib.load()
    src = _fortran_device(SRC, torch.complex64)
    S, Nx, Ny = src.shape
    blocks = [_colmajor2d(b) for b in (Ld, Ll, Lu, Ud, Ul, Uu)]
    inv = invT.permute(2, 1, 0).contiguous() if invT.dim() == 3 else invT
    u = torch.empty_like(src)
    st = stream or torch.cuda.current_stream()
    check(lib.wust_apply_block_lu(C.c_void_p(src.data_ptr()), Ny, Nx, S, *[C.c_void_p(b.data_ptr()) for b in blocks],
                                  C.c_void_p(inv.data_ptr()), int(bool(adjoint)), C.c_void_p(u.data_ptr()),
                                  C.c_void_p(st.cuda_stream)))
    return u.permute(2, 1, 0)


def _colmajor2d(b) -> torch.Tensor:
    """(rows, cols) array -> CUDA complex64 tensor whose memory is column-major."""
    t = b if isinstance(b, torch.Tensor) else torch.as_tensor(np.asarray(b))
    t = t.to(device="cuda", dtype=torch.complex64)
    if t.dim() == 1:
        t = t.unsqueeze(1)
    return t.t().contiguous()
