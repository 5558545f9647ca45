"""B200 (sm_100a) implementation of the WaveformInversionUST Helmholtz gradient path.

The compute lives in ``libwust_b200.so`` (C ABI, include/wust_b200.h); this
package is its Python face: the HelmholtzSolver class, the decompBlockLU /
applyBlockLU drop-ins, the per-frequency oracle and curvature, the NCG
reconstruction loop and a torch.autograd.Function over the misfit.
"""
from ._lib import WustError, load as load_library  # noqa: F401

__all__ = ["WustError", "load_library", "HelmholtzSolver", "decompBlockLU", "applyBlockLU", "Observations",
           "wust_oracle", "directional_curvature", "wust_reconstruct", "misfit"]


def __getattr__(name):
    if name in ("HelmholtzSolver", "decompBlockLU", "applyBlockLU"):
        from . import solver
        return getattr(solver, name)
    if name in ("Observations", "wust_oracle", "directional_curvature"):
        from . import objective
        return getattr(objective, name)
    if name == "wust_reconstruct":
        from .reconstruct import wust_reconstruct
        return wust_reconstruct
    if name == "misfit":
        from .autograd import misfit
        return misfit
    raise AttributeError(name)
