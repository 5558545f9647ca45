"""ctypes binding of libwust_b200.so (declared in include/wust_b200.h).

The shared library is the product; this module only loads it and declares
the C signatures.  There is no fallback: if the library is missing or fails
to load, importing the package's compute API raises.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libwust_b200.so")

WUST_OK = 0
STATUS_NAMES = {
    0: "WUST:OK", 1: "WUST:InvalidInput", 2: "WUST:InvalidOutput", 3: "WUST:CUDAError",
    4: "WUST:CUBLASError", 5: "WUST:CUSOLVERError", 6: "WUST:SingularSchurBlock",
    7: "WUST:InvalidSolverArgument", 8: "WUST:ResourceCleanup", 9: "WUST:RuntimeError",
    10: "WUST:NumericalFailure", 11: "WUST:DeviceTimeout", 12: "WUST:RefinementNotConverged",
}

PRECISION = {"c64": 0, "c64-refined": 1, "bf16-refined": 2, "tf32-refined": 3}
NEED_GRADIENT = 1
RETAIN_STATE = 2

# Symbols that include/wust_b200.h declares (checked by the CPU tests).
EXPORTED = (
    "wust_status_id", "wust_last_error", "wust_version",
    "wust_decomp_block_lu", "wust_decomp_block_lu_noalloc", "wust_apply_block_lu",
    "wust_solver_create", "wust_solver_refactor", "wust_solver_destroy", "wust_solver_timings",
    "wust_solver_stencil", "wust_solver_block", "wust_solver_solve", "wust_solver_mass_apply",
    "wust_solver_oracle", "wust_solver_curvature", "wust_solver_gauss_newton_product", "wust_ncg_roi_gradient", "wust_ncg_direction",
    "wust_ncg_dot", "wust_ncg_project", "wust_dtft", "wust_simulate", "wust_solver_stats", "wust_solver_factor_stats", "wust_solver_factor_info", "wust_solver_sweep_times",
    "wust_selftest_barrier_timeout",
)


class WustError(RuntimeError):
    """A failing library call; ``identifier`` is the reference error id."""

    def __init__(self, status: int, message: str):
        self.status = status
        self.identifier = STATUS_NAMES.get(status, "WUST:Unknown")
        super().__init__(f"{self.identifier}: {message}")


class SolverOptions(C.Structure):
    _fields_ = [
        ("ny", C.c_int), ("nx", C.c_int),
        ("x_m", C.POINTER(C.c_double)), ("y_m", C.POINTER(C.c_double)),
        ("frequency_hz", C.c_double), ("sign_convention", C.c_double),
        ("pml_strength", C.c_double), ("pml_m", C.c_double),
        ("stencil_vmin", C.c_double), ("stencil_vmax", C.c_double),
        ("dispersion", C.c_int), ("time_step_s", C.c_double), ("reference_speed_mps", C.c_double),
        ("precision", C.c_int), ("refine_max_iters", C.c_int), ("refine_tol", C.c_double),
        ("max_sources", C.c_int), ("factor_method", C.c_int), ("sweep_method", C.c_int), ("correction_precision", C.c_int),
        ("max_ctas", C.c_int), ("chunk_count", C.c_int),
    ]


_lib = None


def load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m waveforminversionust_b200.build`")
    lib = C.CDLL(LIB_PATH)
    vp, i, d = C.c_void_p, C.c_int, C.c_double
    pd, pi = C.POINTER(C.c_double), C.POINTER(C.c_int)
    lib.wust_status_id.restype = C.c_char_p
    lib.wust_status_id.argtypes = [i]
    lib.wust_last_error.restype = C.c_char_p
    lib.wust_last_error.argtypes = []
    lib.wust_version.argtypes = [pi, pi, pi]
    lib.wust_decomp_block_lu.argtypes = [vp] * 9 + [i, i, vp, C.POINTER(C.c_float), vp]
    lib.wust_decomp_block_lu_noalloc.argtypes = [vp] * 9 + [i, i, vp, vp]
    lib.wust_apply_block_lu.argtypes = [vp, i, i, i] + [vp] * 7 + [i, vp, vp]
    lib.wust_solver_create.argtypes = [C.POINTER(vp), C.POINTER(SolverOptions), vp, vp, vp]
    lib.wust_solver_refactor.argtypes = [vp, vp, vp, d]
    lib.wust_solver_destroy.argtypes = [vp]
    lib.wust_solver_timings.argtypes = [vp, pd, pd]
    lib.wust_solver_stencil.argtypes = [vp, pd, pd, pd]
    lib.wust_solver_block.argtypes = [vp, C.c_char_p, C.POINTER(vp), pi, pi, pi]
    lib.wust_solver_solve.argtypes = [vp, vp, i, i, vp, vp]
    lib.wust_solver_mass_apply.argtypes = [vp, vp, i, i, vp]
    lib.wust_solver_oracle.argtypes = [vp, vp, i, vp, i, vp, vp, i, i, pd, vp]
    lib.wust_solver_curvature.argtypes = [vp, vp, pd]
    lib.wust_solver_gauss_newton_product.argtypes = [vp, vp, vp, pd]
    d = C.c_double
    lib.wust_ncg_roi_gradient.argtypes = [vp, vp, vp, d, d, d, d, vp, vp]
    lib.wust_ncg_direction.argtypes = [vp, vp, vp, vp, d, C.c_int, vp, pd, pd]
    lib.wust_ncg_dot.argtypes = [vp, vp, vp, pd]
    lib.wust_ncg_project.argtypes = [vp, vp, vp, d, d, d, d, d, vp, pd]
    lib.wust_dtft.argtypes = [vp, i, vp, i, vp, i, i, i, vp, vp, vp]
    lib.wust_simulate.argtypes = [vp, i, i, d, d, d, i, vp, vp, i, vp, i, i, d, d, i, i, vp, vp]
    lib.wust_solver_stats.argtypes = [vp, pi, pd, pd, C.POINTER(C.c_longlong)]
    lib.wust_solver_factor_stats.argtypes = [vp, C.POINTER(C.c_longlong)]
    lib.wust_solver_factor_info.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    lib.wust_solver_sweep_times.argtypes = [vp, pd, C.POINTER(C.c_longlong)]
    lib.wust_selftest_barrier_timeout.argtypes = [i, pi]
    for name in EXPORTED:
        if name not in ("wust_status_id", "wust_last_error"):
            getattr(lib, name).restype = i
    _lib = lib
    return lib


def check(status: int) -> None:
    if status != WUST_OK:
        msg = load().wust_last_error().decode(errors="replace")
        raise WustError(status, msg)
