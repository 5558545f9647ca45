"""wust_decomp_block_lu_noalloc: the factorization for callers that cannot allocate.

Hosts that own the device heap (MATLAB's gpuArray manager, framework caching
allocators) or that cannot pay cudaMalloc's device synchronization use this
entry point; its scratch is a static device array, so it allocates nothing.
The test calls it through the C ABI twice in a row on different operators
and checks each result against the allocating entry point
(wust_decomp_block_lu) with the tolerance the factor parity tests use.
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
