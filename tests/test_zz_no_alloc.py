"""wust_decomp_block_lu_noalloc: the factorization for callers that cannot allocate.

Hosts that own the device heap (MATLAB's gpuArray manager, framework caching
allocators) or that cannot pay cudaMalloc's device synchronization use this
entry point; its scratch is a static device array, so it allocates nothing.
The tests call it through the C ABI twice in a row on different operators
and once at its largest grid, and check each result against the allocating
entry point (wust_decomp_block_lu) with the tolerance the factor parity
tests use; the largest-grid test also checks that the device's free memory
does not change across a call.
The file name makes pytest collect it last.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]

NAMES = ("Ld", "Ll", "Lu", "Dd", "Dl", "Du", "Ud", "Ul", "Uu")


def _blocks(p, c, f):
    from oracle import helmholtz_fp64 as o
    s = o.HelmholtzSolverFP64(p.x_m, p.y_m, c, np.zeros(p.shape), f, -1, 10.0, p.pml_m,
                              dict(backend="cpu", stencil_bounds=(1400, 1700)), factor=False)
    return s.coefs


def _device_colmajor(a):
    import torch
    return torch.as_tensor(np.asarray(a, np.complex64).T.copy(), device="cuda")


def _factor(lib, fn, coefs, noalloc):
    import torch
    ny, nx = coefs["Dd"].shape
    dev = [_device_colmajor(coefs[n]) for n in NAMES]
    invT = torch.full((nx, ny, ny), complex(np.nan, np.nan), dtype=torch.complex64, device="cuda")
    args = [C.c_void_p(t.data_ptr()) for t in dev] + [ny, nx, C.c_void_p(invT.data_ptr())]
    if noalloc:
        rc = fn(*args, None)
    else:
        rc = fn(*args, None, None)
    torch.cuda.synchronize()
    return rc, invT.cpu().numpy()


def test_noalloc_matches_allocating_entry_point_twice():
    from waveforminversionust_b200 import _lib
    from waveforminversionust_b200 import synthetic
    lib = _lib.load()
    p = synthetic.small(seed=5)
    ops = [_blocks(p, p.c_true, 0.3e6), _blocks(p, p.c_init, 0.4e6)]
    for coefs in ops:                     # two calls in a row share the static scratch
        rc, got = _factor(lib, lib.wust_decomp_block_lu_noalloc, coefs, noalloc=True)
        assert rc == 0, lib.wust_last_error().decode()
        rc, want = _factor(lib, lib.wust_decomp_block_lu, coefs, noalloc=False)
        assert rc == 0, lib.wust_last_error().decode()
        assert np.all(np.isfinite(got))
        err = np.linalg.norm(got - want) / np.linalg.norm(want)
        assert err < 2e-5


def _dominant_blocks(ny, nx, seed):
    """A diagonally dominant block-tridiagonal operator in the reference's
    nine block shapes (every Schur page well conditioned)."""
    rng = np.random.default_rng(seed)

    def c(shape, scale, offset=0.0):
        return offset + scale * (rng.standard_normal(shape) + 1j * rng.standard_normal(shape))
    return dict(Dd=c((ny, nx), 0.1, 4.0), Dl=c((ny - 1, nx), 0.2, -1.0), Du=c((ny - 1, nx), 0.2, -1.0),
                Ld=c((ny, nx - 1), 0.1, -0.5), Ll=c((ny - 1, nx - 1), 0.05), Lu=c((ny - 1, nx - 1), 0.05),
                Ud=c((ny, nx - 1), 0.1, -0.5), Ul=c((ny - 1, nx - 1), 0.05), Uu=c((ny - 1, nx - 1), 0.05))


def test_noalloc_at_its_largest_grid_matches_and_allocates_nothing():
    """At Ny = WUST_NOALLOC_MAX_NY the static scratch is used to its last
    byte; the result must still match the allocating entry point, and the
    device's free memory must not move across a call (nothing allocated)."""
    import torch
    from waveforminversionust_b200 import _lib
    lib = _lib.load()
    ny, nx = 1024, 3
    coefs = _dominant_blocks(ny, nx, seed=11)
    rc, want = _factor(lib, lib.wust_decomp_block_lu, coefs, noalloc=False)
    assert rc == 0, lib.wust_last_error().decode()
    dev = [_device_colmajor(coefs[n]) for n in NAMES]
    invT = torch.full((nx, ny, ny), complex(np.nan, np.nan), dtype=torch.complex64, device="cuda")
    args = [C.c_void_p(t.data_ptr()) for t in dev] + [ny, nx, C.c_void_p(invT.data_ptr()), None]
    assert lib.wust_decomp_block_lu_noalloc(*args) == 0, lib.wust_last_error().decode()   # warm-up
    torch.cuda.synchronize()
    invT.fill_(complex(np.nan, np.nan))
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    rc = lib.wust_decomp_block_lu_noalloc(*args)
    torch.cuda.synchronize()
    free_after = torch.cuda.mem_get_info()[0]
    assert rc == 0, lib.wust_last_error().decode()
    assert free_after == free_before, (free_before, free_after)
    got = invT.cpu().numpy()
    assert np.all(np.isfinite(got))
    err = np.linalg.norm(got - want) / np.linalg.norm(want)
    assert err < 2e-5


def test_noalloc_rejects_grids_beyond_its_limit():
    import torch
    from waveforminversionust_b200 import _lib
    lib = _lib.load()
    ny, nx = 1025, 4
    dummy = torch.zeros(16, dtype=torch.complex64, device="cuda")
    ptr = C.c_void_p(dummy.data_ptr())
    rc = lib.wust_decomp_block_lu_noalloc(*([ptr] * 9), ny, nx, ptr, None)
    assert rc == 1
    assert "1024" in lib.wust_last_error().decode()
