"""GPU tests of the NCG update on the device (wust_ncg_* through the C ABI):
each rule against its NumPy restatement of wust_reconstruct.m:24-57, and the
device-resident reconstruction loop against the host loop."""
import ctypes as C

import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]


def rel(a, b):
    return np.linalg.norm(np.ravel(a - b)) / max(np.linalg.norm(np.ravel(b)), 1e-300)


@pytest.fixture(scope="module", params=[(40, 52), (31, 31)], ids=["even-40x52", "odd-31x31"])
def grid(request):
    from waveforminversionust_b200.solver import HelmholtzSolver
    ny, nx = request.param
    x = (np.arange(nx) - (nx - 1) / 2) * 3e-4
    y = (np.arange(ny) - (ny - 1) / 2) * 2.5e-4
    s = HelmholtzSolver(x, y, np.full((ny, nx), 1500.0), None, 5e5, -1, 10.0, 4 * 3e-4,
                        dict(backend="gpu", stencil_bounds=(1400, 1700)))
    yield s, x, y
    s.close()


def _dev(a, dtype=None):
    import torch
    return torch.as_tensor(np.ascontiguousarray(np.asarray(a).T), dtype=dtype, device="cuda")


def _host(t):
    return t.cpu().numpy().T


def _p(t):
    return C.c_void_p(t.data_ptr())


def test_roi_filter_direction_dot_and_projection_match_numpy(grid):
    import torch
    from waveforminversionust_b200 import _lib
    from waveforminversionust_b200._lib import check
    from waveforminversionust_b200.ncg import (linearized_step_length, ncg_direction, project_slowness_update,
                                               roi_gradient)
    s, x, y = grid
    lib = _lib.load()
    h = C.c_void_p(s.handle)
    ny, nx = s.shape
    rng = np.random.default_rng(7)
    g = rng.standard_normal((ny, nx))
    mask = np.zeros((ny, nx), bool)
    mask[3:-4, 5:-3] = True
    g_d, m_d = _dev(g, torch.float64), _dev(mask.astype(np.uint8), torch.uint8)
    roi_d, z_d = torch.empty_like(g_d), torch.empty_like(g_d)
    for cutoff, order in ((0.0, 4.0), (0.6, 4.0), (1.3, 2.5)):
        check(lib.wust_ncg_roi_gradient(h, _p(g_d), _p(m_d), 1480.0, 7e5, cutoff, order, _p(roi_d), _p(z_d)))
        roi, z = roi_gradient(g, mask, x, y, 1480.0, 7e5, cutoff, order)
        assert np.array_equal(_host(roi_d), roi)
        assert rel(_host(z_d), z) < 1e-12, cutoff
        if cutoff > 0:
            assert rel(z, roi) > 1e-3               # the filter did something
    # direction: PR/FR clipping, a different frequency, and the restart on non-descent
    z_prev = rng.standard_normal((ny, nx)) * mask
    d_prev = rng.standard_normal((ny, nx)) * mask
    for same, prev_gz, dprev in ((True, 3.0, d_prev), (False, 3.0, d_prev), (True, 1e-3, 50 * z)):
        dd = _dev(dprev, torch.float64)
        beta, gz = C.c_double(), C.c_double()
        check(lib.wust_ncg_direction(h, _p(roi_d), _p(z_d), _p(_dev(z_prev, torch.float64)), prev_gz, int(same),
                                     _p(dd), C.byref(beta), C.byref(gz)))
        d_ref, beta_ref, gz_ref = ncg_direction(roi, z, z_prev, prev_gz, dprev, same)
        assert rel(_host(dd), d_ref) < 1e-12 and abs(beta.value - beta_ref) <= 1e-12 * max(1, abs(beta_ref))
        assert abs(gz.value - gz_ref) <= 1e-12 * abs(gz_ref)
    assert beta.value == 0.0                       # the last case is not a descent direction: restart with -z
    slope = C.c_double()
    check(lib.wust_ncg_dot(h, _p(roi_d), _p(dd), C.byref(slope)))
    assert abs(slope.value - float(np.sum(roi * d_ref))) <= 1e-12 * abs(float(np.sum(roi * d_ref)))
    # projection: small and large steps (the speed clip binds), update mask
    c = 1500 + 30 * rng.standard_normal((ny, nx))
    cfg = dict(max_update_mps=12.0, bounds_mps=(1400.0, 1600.0), step_damping=0.8, update_mask=mask)
    for alpha in (linearized_step_length(-1e-6, 1.0), 1e-3):
        c_d = _dev(c, torch.float64)
        rel_u = C.c_double()
        check(lib.wust_ncg_project(h, _p(c_d), _p(dd), alpha, 0.8, 12.0, 1400.0, 1600.0, _p(m_d), C.byref(rel_u)))
        c_ref = project_slowness_update(c, d_ref, alpha, cfg)
        assert rel(_host(c_d), c_ref) < 1e-14
        ref_u = np.linalg.norm((1 / c_ref)[mask] - (1 / c)[mask]) / np.linalg.norm((1 / c)[mask])
        assert abs(rel_u.value - ref_u) <= 1e-10 * ref_u
    with pytest.raises(Exception):
        check(lib.wust_ncg_roi_gradient(h, _p(g_d), _p(m_d), 1480.0, 7e5, -1.0, 4.0, _p(roi_d), _p(z_d)))


def test_device_reconstruction_matches_host_loop(ref_fixture):
    """Three NCG updates (two frequencies, with the ringing filter) of the
    device-resident loop against the host loop.  The first oracle call sees
    identical inputs; the filtered gradients differ by FFT rounding (1e-13),
    which the complex-single curvature solve can carry to 1e-8; later updates
    agree to the refined solves' 1e-5."""
    from waveforminversionust_b200.objective import POOL, Observations
    from waveforminversionust_b200.reconstruct import wust_reconstruct
    fx = ref_fixture
    o = fx["obs"]
    obs = Observations(o.x_m, o.y_m, o.tx_index, o.rx_index, o.frequencies_hz, o.Y, o.mask)
    base = dict(backend="gpu", bounds_mps=(1300.0, 1800.0), max_update_mps=12.0, step_damping=1.0,
                source_batch_size=2, pml_strength=10.0, pml_m=.004, stencil_bounds=(1400.0, 1700.0),
                wavenumber="continuum", filter_cutoff=0.8, filter_order=4, update_mask=fx["mask"].astype(float),
                frequency_schedule_hz=[1e5, 1e5, 1.2e5], precision="c64-refined", save_history=True)
    out = {}
    for dev in (False, True):
        POOL.clear()
        out[dev] = wust_reconstruct(obs, fx["initial"], dict(base, ncg_device=dev))
    POOL.clear()
    rh, rd = out[False]["records"], out[True]["records"]
    assert len(rh) == len(rd) == 3
    assert rd[0]["loss_before_update"] == rh[0]["loss_before_update"]
    for k in ("alpha", "beta", "curvature", "relative_slowness_update"):
        assert abs(rd[0][k] - rh[0][k]) <= 1e-7 * max(abs(rh[0][k]), 1e-30), k
    assert rel(out[True]["history_mps"][:, :, 1], out[False]["history_mps"][:, :, 1]) < 1e-9
    for a, b in zip(rd, rh):
        for k in ("loss_before_update", "alpha", "curvature"):
            assert abs(a[k] - b[k]) <= 1e-5 * abs(b[k]), (a["step"], k)
    assert rel(1 / out[True]["c_mps"], 1 / out[False]["c_mps"]) < 1e-7
    assert rd[2]["loss_before_update"] < rd[0]["loss_before_update"]
