"""GPU tests of the library's callers: the autograd misfit, the k-Wave LDR-9
dispersion option and the NCG reconstruction loop, each against the FP64
oracle or its defining property (calls go through the C ABI)."""
import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]


def _gpu_obs(o_obs):
    from waveforminversionust_b200.objective import Observations
    return Observations(o_obs.x_m, o_obs.y_m, o_obs.tx_index, o_obs.rx_index, o_obs.frequencies_hz, o_obs.Y,
                        o_obs.mask)


@pytest.mark.parametrize("precision", ["c64-refined", "tf32-refined"])
def test_autograd_misfit_matches_central_differences(ref_fixture, precision):
    """torch.autograd over Phi_f(s): backward (adjoint solve + slowness
    gradient, factors reused) against central differences at relative steps
    1e-3 .. 1e-5, FP64 tolerance 1e-4 (test_runtime.m:45-56)."""
    import torch
    from waveforminversionust_b200.autograd import misfit
    from waveforminversionust_b200.objective import POOL, default_config
    fx = ref_fixture
    obs = _gpu_obs(fx["obs"])
    cfg = default_config(pml_m=.004, pml_strength=10, source_batch_size=2, precision=precision, refine_tol=1e-10)
    s0 = torch.tensor(1 / fx["initial"], dtype=torch.float64, device="cuda", requires_grad=True)
    loss = misfit(s0, obs, 0, cfg)
    loss.backward()
    d = torch.tensor(fx["direction"], dtype=torch.float64, device="cuda")
    adj = float((s0.grad * d).sum())
    for rel_step in (1e-3, 1e-4, 1e-5):
        h = rel_step * float(s0.detach().abs().max()) / float(d.abs().max())
        with torch.no_grad():
            lp = float(misfit(s0.detach() + h * d, obs, 0, cfg))
            lm = float(misfit(s0.detach() - h * d, obs, 0, cfg))
        fd = (lp - lm) / (2 * h)
        assert abs(fd - adj) / max(abs(fd), abs(adj)) < 1e-4, (rel_step, fd, adj)
    POOL.clear()


def test_ldr9_dispersion_matches_oracle(ref_fixture):
    """wavenumber='kwave-ldr9' (kwaveLdr9WavenumberSquared.m) on the GPU: the
    refined misfit and gradient equal the FP64 oracle's."""
    from oracle import helmholtz_fp64 as o
    from waveforminversionust_b200.objective import POOL, default_config, wust_oracle
    fx = ref_fixture
    disp = dict(time_step_s=2e-8, reference_speed_mps=1700)
    cfg_o = o.OracleConfig(pml_m=.004, source_batch_size=2, wavenumber="kwave-ldr9", dispersion=disp)
    loss_ref, grad_ref, _ = o.wust_oracle(fx["initial"], fx["obs"], 0, cfg_o)
    cfg = default_config(pml_m=.004, pml_strength=10, source_batch_size=2, precision="c64-refined", refine_tol=1e-10,
                         wavenumber="kwave-ldr9", dispersion=disp)
    loss, grad = wust_oracle(fx["initial"], _gpu_obs(fx["obs"]), 0, cfg)
    assert abs(loss - loss_ref) / loss_ref < 1e-7
    assert np.linalg.norm(grad - grad_ref) / np.linalg.norm(grad_ref) < 1e-5
    # the dispersion option changes the operator (it is not silently ignored)
    loss_cont, _ = wust_oracle(fx["initial"], _gpu_obs(fx["obs"]), 0,
                               default_config(pml_m=.004, pml_strength=10, source_batch_size=2,
                                              precision="c64-refined", refine_tol=1e-10))
    assert abs(loss_cont - loss) / loss > 1e-6
    POOL.clear()


def test_reconstruction_descends_and_matches_oracle_first_step(ref_fixture):
    """Three NCG updates of wust_reconstruct (wust_reconstruct.m:20-74) at one
    frequency on the GPU: the misfit before each update decreases, and the
    first misfit equals the FP64 oracle's."""
    from oracle import helmholtz_fp64 as o
    from waveforminversionust_b200.objective import POOL
    from waveforminversionust_b200.reconstruct import wust_reconstruct
    fx = ref_fixture
    obs = _gpu_obs(fx["obs"])
    cfg = dict(backend="gpu", bounds_mps=(1300.0, 1800.0), max_update_mps=12.0, step_damping=1.0,
               source_batch_size=2, pml_strength=10.0, pml_m=.004, stencil_bounds=(1400.0, 1700.0),
               wavenumber="continuum", filter_cutoff=0.0, filter_order=4, update_mask=fx["mask"].astype(float),
               frequency_schedule_hz=[1e5, 1e5, 1e5], precision="c64-refined")
    out = wust_reconstruct(obs, fx["initial"], cfg)
    losses = [r["loss_before_update"] for r in out["records"]]
    assert len(losses) == 3 and losses[1] < losses[0] and losses[2] < losses[1], losses
    loss0, _, _ = o.wust_oracle(fx["initial"], fx["obs"], 0, fx["cfg"], need_gradient=False)
    assert abs(losses[0] - loss0) / loss0 < 1e-5
    assert all(r["curvature"] > 0 and r["alpha"] >= 0 for r in out["records"])
    POOL.clear()


@pytest.fixture(scope="module")
def small():
    from waveforminversionust_b200 import synthetic
    return synthetic.small(seed=3), None


def test_tensor_core_profile_edge_cases(small):
    """TF32 profile: an all-zero right-hand side returns zeros, a single
    source agrees with the c64 refined profile, more sources than one call
    holds are batched, and grids beyond the tensor-core tiling are rejected
    with WUST:InvalidInput."""
    from waveforminversionust_b200._lib import WustError
    from waveforminversionust_b200.solver import HelmholtzSolver
    p, ref = small
    ny, nx = p.shape
    opts = dict(backend="gpu", stencil_bounds=(1400, 1700))
    f = p.frequencies_hz[0]
    tc = HelmholtzSolver(p.x_m, p.y_m, p.c_true, None, f, -1, 10.0, p.pml_m, opts, precision="tf32-refined",
                         max_sources=4)
    z = tc.solve(np.zeros((ny, nx, 3), np.complex64)).cpu().numpy()
    assert np.all(z == 0)
    rng = np.random.default_rng(2)
    b = np.zeros((ny, nx, 1), np.complex64)
    b[1:-1, 1:-1, 0] = rng.standard_normal((ny - 2, nx - 2)) + 1j * rng.standard_normal((ny - 2, nx - 2))
    c64 = HelmholtzSolver(p.x_m, p.y_m, p.c_true, None, f, -1, 10.0, p.pml_m, opts, precision="c64-refined",
                          max_sources=4)
    for adjoint in (False, True):
        a = tc.solve(b, adjoint=adjoint).cpu().numpy()[1:-1, 1:-1]
        w = c64.solve(b, adjoint=adjoint).cpu().numpy()[1:-1, 1:-1]
        assert np.linalg.norm(a - w) / np.linalg.norm(w) < 3e-5, adjoint
    # more sources than one call holds: the Python solver batches them
    b5 = np.repeat(b, 5, axis=2)
    u5 = tc.solve(b5).cpu().numpy()
    u1 = tc.solve(b).cpu().numpy()
    assert np.linalg.norm(u5 - u1) / np.linalg.norm(u1) < 1e-6
    tc.close()
    c64.close()
    n = 600                                   # beyond the 4 x 9 x 16-row tensor-core K tiling
    xg = (np.arange(n) - (n - 1) / 2) * 3e-4
    with pytest.raises(WustError) as e:
        HelmholtzSolver(xg, xg, np.full((n, n), 1500.0), None, 5e5, -1, 10.0, 16 * 3e-4, opts,
                        precision="tf32-refined", max_sources=4)
    assert e.value.identifier == "WUST:InvalidInput"


@pytest.mark.parametrize("precision", ["c64-refined", "tf32-refined"])
def test_reconstruction_final_sound_speed_matches_oracle(precision):
    """Four NCG updates over two frequencies (wust_reconstruct.m:20-74) on an
    80 x 80 grid with 8 transmitters and a 32-element ring: the final sound
    speed of the device loop is within 0.5 m/s RMS of the FP64 oracle's
    reconstruction (the accuracy bar of the refined solver), asserted with a
    tenfold margin, after the reconstruction moved the model by more than 1 m/s."""
    from oracle import helmholtz_fp64 as o
    from waveforminversionust_b200 import synthetic
    from waveforminversionust_b200.objective import POOL
    from waveforminversionust_b200.reconstruct import wust_reconstruct
    p = synthetic._problem("recon80", 64, 8, 0.5e-3, 32, 14e-3, 8, [0.25e6, 0.35e6],
                           lambda X, Y: 1500 + 25 * np.exp(-((X - 2e-3) ** 2 + Y ** 2) / (2 * (4e-3) ** 2)), 12e-3)
    ny, nx = p.shape
    ocfg = o.OracleConfig(pml_m=p.pml_m, pml_strength=10, stencil_bounds=(1400, 1700), source_batch_size=4)
    nf = p.frequencies_hz.size
    n_tx, n_rx = p.tx_index.size, p.rx_index.size
    dummy = o.Observations(p.x_m, p.y_m, p.tx_index, p.rx_index, p.frequencies_hz, np.zeros((n_tx, n_rx, nf)),
                           np.ones((n_tx, n_rx, nf), bool))
    Y = np.zeros((n_tx, n_rx, nf), complex)
    for fi in range(nf):
        u = o.make_solver(p.c_true, dummy, fi, ocfg).solve(o.point_sources(p.tx_index, range(n_tx), ny, nx))
        Y[:, :, fi] = u.reshape(-1, n_tx, order="F")[p.rx_index - 1, :].T
    obs = o.Observations(p.x_m, p.y_m, p.tx_index, p.rx_index, p.frequencies_hz, Y, np.ones((n_tx, n_rx, nf), bool))
    schedule = [0, 0, 1, 1]
    bounds, max_update, damping = (1400.0, 1700.0), 12.0, 1.0
    # the FP64 oracle's loop
    c = p.c_init.copy()
    mask = p.update_mask
    prev_z, prev_gz, direction, last = np.zeros_like(c), 0.0, np.zeros_like(c), None
    for fi in schedule:
        _, g, state = o.wust_oracle(c, obs, fi, ocfg, need_gradient=True, retain_state=True)
        roi, z = o.roi_gradient(g, mask, p.x_m, p.y_m, 1500.0, p.frequencies_hz[fi], 0.0, 4)
        direction, _, gz = o.ncg_direction(roi, z, prev_z, prev_gz, direction, fi == last)
        prev_z, prev_gz, last = z, gz, fi
        curvature = o.directional_curvature(state, direction, obs.rx_index, obs.mask[:, :, fi])
        alpha = o.linearized_step_length(float(np.sum(roi * direction)), curvature)
        c = o.project_slowness_update(c, direction, alpha, max_update, bounds, damping, mask)
    # the device loop
    cfg = dict(backend="gpu", bounds_mps=bounds, max_update_mps=max_update, step_damping=damping,
               source_batch_size=4, pml_strength=10.0, pml_m=p.pml_m, stencil_bounds=(1400.0, 1700.0),
               wavenumber="continuum", filter_cutoff=0.0, filter_order=4, update_mask=mask.astype(float),
               frequency_schedule_hz=[p.frequencies_hz[k] for k in schedule], precision=precision)
    out = wust_reconstruct(_gpu_obs(obs), p.c_init, cfg)
    POOL.clear()
    rms = float(np.sqrt(np.mean((out["c_mps"] - c) ** 2)))
    assert float(np.sqrt(np.mean((c - p.c_init) ** 2))) > 1.0
    assert rms < 0.05, rms


def test_autograd_forward_only_and_gauss_newton_products(ref_fixture):
    """The Function on a device slowness: without requires_grad it runs the
    forward solve only (fewer sweeps, same misfit); with create_graph its
    gradient is differentiable and torch.autograd gives the Gauss-Newton
    Hessian-vector product, matching the FP64 oracle's and reproducing
    directional_curvature as its quadratic form."""
    import torch
    from oracle import helmholtz_fp64 as o
    from waveforminversionust_b200.autograd import misfit
    from waveforminversionust_b200.objective import POOL, default_config
    fx = ref_fixture
    obs = _gpu_obs(fx["obs"])
    cfg = default_config(pml_m=.004, pml_strength=10, source_batch_size=3, precision="c64-refined", refine_tol=1e-10)
    s = torch.tensor(1 / fx["initial"], dtype=torch.float64, device="cuda")
    l0 = misfit(s, obs, 0, cfg)                         # no gradient wanted: forward only
    solver = next(iter(POOL._pool.values()))
    n0 = solver.sweep_times()[1]
    l1 = misfit(s, obs, 0, cfg)
    pairs_forward = solver.sweep_times()[1] - n0
    s1 = s.clone().requires_grad_(True)
    n0 = solver.sweep_times()[1]
    l2 = misfit(s1, obs, 0, cfg)
    pairs_gradient = solver.sweep_times()[1] - n0
    assert float(l0) == float(l1) and abs(float(l2.detach()) - float(l1)) <= 1e-12 * float(l1)
    assert 0 < pairs_forward < pairs_gradient, (pairs_forward, pairs_gradient)
    (g,) = torch.autograd.grad(l2, s1, create_graph=True)
    assert g.is_cuda
    d = torch.tensor(fx["direction"], dtype=torch.float64, device="cuda")
    e = torch.roll(d, 3, dims=1) * torch.tensor(fx["mask"], dtype=torch.float64, device="cuda")
    (hd,) = torch.autograd.grad(g, s1, d, retain_graph=True)
    (he,) = torch.autograd.grad(g, s1, e)
    _, g_ref, state = o.wust_oracle(fx["initial"], fx["obs"], 0, fx["cfg"], retain_state=True)
    hd_ref, k_ref = o.gauss_newton_product(state, fx["direction"], fx["obs"].rx_index, fx["obs"].mask[:, :, 0])
    assert np.linalg.norm(g.detach().cpu().numpy() - g_ref) <= 1e-5 * np.linalg.norm(g_ref)
    hd_np = hd.cpu().numpy()
    assert np.linalg.norm(hd_np - hd_ref) <= 1e-5 * np.linalg.norm(hd_ref)
    assert abs(float((d * hd).sum()) - k_ref) <= 1e-5 * k_ref
    assert abs(float((e * hd).sum()) - float((d * he).sum())) <= 1e-6 * abs(float((d * hd).sum()))
    POOL.clear()
