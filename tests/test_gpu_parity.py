"""GPU parity of libwust_b200 against the FP64 oracle (calls go through the C ABI).

Tolerances: complex-single block LU ("c64", the reference's GPU algorithm)
is compared at single-precision accuracy scaled by the conditioning of the
operator; the refined profile must reach 1e-5 relative pressure error and
1e-4 gradient error against the FP64 sparse LU (the targets of the path).
"""
import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(np.asarray(b).ravel()), 1e-300))


def to_np(t):
    return t.detach().cpu().numpy()


@pytest.fixture(scope="module")
def small():
    from waveforminversionust_b200 import synthetic
    from oracle import helmholtz_fp64 as o
    p = synthetic.small(seed=3)
    solver = o.HelmholtzSolverFP64(p.x_m, p.y_m, p.c_true, np.zeros(p.shape), p.frequencies_hz[0], -1, 10.0,
                                   p.pml_m, dict(backend="cpu", stencil_bounds=(1400, 1700)))
    return p, solver


def make_gpu_solver(p, c, f, precision="c64", max_sources=64):
    from waveforminversionust_b200.solver import HelmholtzSolver
    return HelmholtzSolver(p.x_m, p.y_m, c, None, f, -1, 10.0, p.pml_m,
                           dict(backend="gpu", stencil_bounds=(1400, 1700)), precision=precision,
                           max_sources=max_sources)


def test_assembly_matches_oracle(small):
    p, ref = small
    s = make_gpu_solver(p, p.c_true, p.frequencies_hz[0])
    assert abs(s.massD - ref.d) < 1e-12 and abs(s.massE - ref.e) < 1e-12
    for name in ("Dd", "Dl", "Du", "Ld", "Ll", "Lu", "Ud", "Ul", "Uu"):
        got = to_np(s.block(name)).astype(np.complex128)
        want = ref.coefs[name]
        assert got.shape == want.shape, name
        assert rel(got, want) < 1e-6, name
        # structure: zeros where the reference leaves zeros
        assert np.all((np.abs(want) == 0) == (np.abs(got) == 0)), name
    mult = to_np(s.block("mult"))
    assert rel(mult, ref.virtual_source_multiplier) < 1e-12
    s.close()


def test_factor_matches_oracle_block_lu(small):
    from oracle import helmholtz_fp64 as o
    p, ref = small
    s = make_gpu_solver(p, p.c_true, p.frequencies_hz[0])
    invT = to_np(s.block("invT")).astype(np.complex128)
    want = o.block_lu_factor(ref.coefs)
    assert invT.shape == want.shape
    # border rows/columns are exactly zero (decompBlockLU.cu:284-288)
    assert np.all(invT[[0, -1], :, :] == 0) and np.all(invT[:, [0, -1], :] == 0)
    assert rel(invT, want) < 2e-5
    s.close()


def test_decomp_and_apply_dropins(small):
    """decompBlockLU / applyBlockLU drop-ins on the reference's 9 blocks."""
    import torch
    from oracle import helmholtz_fp64 as o
    from waveforminversionust_b200.solver import applyBlockLU, decompBlockLU
    p, ref = small
    c = ref.coefs
    invT, timing = decompBlockLU(c["Ld"], c["Ll"], c["Lu"], c["Dd"], c["Dl"], c["Du"], c["Ud"], c["Ul"], c["Uu"],
                                 timings=True)
    want = o.block_lu_factor(c)
    assert rel(to_np(invT), want) < 2e-5
    assert timing["block_count"] == p.shape[1] and timing["total_gpu_ms"] > 0
    rng = np.random.default_rng(0)
    ny, nx = p.shape
    src = rng.standard_normal((ny, nx, 5)) + 1j * rng.standard_normal((ny, nx, 5))
    for adjoint in (False, True):
        got = to_np(applyBlockLU(torch.as_tensor(src.astype(np.complex64)), c["Ld"], c["Ll"], c["Lu"], c["Ud"],
                                 c["Ul"], c["Uu"], invT, adjoint))
        want_u = o.block_lu_apply(src, c, want, adjoint)
        assert rel(got, want_u) < 5e-5, adjoint


def test_solve_matches_sparse_lu(small):
    p, ref = small
    s = make_gpu_solver(p, p.c_true, p.frequencies_hz[0])
    from oracle import helmholtz_fp64 as o
    ny, nx = p.shape
    src = o.point_sources(p.tx_index, range(p.tx_index.size), ny, nx)
    u = to_np(s.solve(src.astype(np.complex64)))
    want = ref.solve(src)
    assert rel(u, want) < 1e-4
    # adjoint: interior agrees with the sparse H^H solve
    rng = np.random.default_rng(1)
    r = np.zeros((ny, nx, 4), complex)
    r[1:-1, 1:-1] = rng.standard_normal((ny - 2, nx - 2, 4)) + 1j * rng.standard_normal((ny - 2, nx - 2, 4))
    lam = to_np(s.solve(r.astype(np.complex64), adjoint=True))
    lam_ref = ref.solve(r, adjoint=True)
    assert rel(lam[1:-1, 1:-1], lam_ref[1:-1, 1:-1]) < 1e-4
    s.close()


@pytest.mark.parametrize("precision", ["c64-refined", "tf32-refined", "bf16-refined"])
def test_refined_solve_reaches_fp64_accuracy(small, precision):
    p, ref = small
    from oracle import helmholtz_fp64 as o
    s = make_gpu_solver(p, p.c_true, p.frequencies_hz[0], precision=precision)
    ny, nx = p.shape
    src = o.point_sources(p.tx_index, range(p.tx_index.size), ny, nx)
    u = to_np(s.solve(src.astype(np.complex64)))
    st = s.stats()
    assert st["refine_iters"] >= 1 and st["error_estimate"] <= 1e-5
    assert rel(u, ref.solve(src)) < 1e-5
    # adjoint solve, interior (the block solver leaves the top/bottom border at zero)
    rng = np.random.default_rng(4)
    ny, nx = p.shape
    r = np.zeros((ny, nx, 3), complex)
    r[1:-1, 1:-1] = rng.standard_normal((ny - 2, nx - 2, 3)) + 1j * rng.standard_normal((ny - 2, nx - 2, 3))
    lam = to_np(s.solve(r.astype(np.complex64), adjoint=True))
    lam_ref = ref.solve(r, adjoint=True)
    assert rel(lam[1:-1, 1:-1], lam_ref[1:-1, 1:-1]) < 1e-5
    s.close()


def test_tensor_core_sweep_split_k_and_source_batches():
    """TF32 tensor-core sweeps on a grid whose K range is split over 4 CTAs,
    with a partial source tile and more sources than one launch holds, agree
    with the complex-single sweeps once both are refined in FP64."""
    from waveforminversionust_b200.solver import HelmholtzSolver
    ny = nx = 330
    dx = 0.3e-3
    x = (np.arange(nx) - (nx - 1) / 2) * dx
    y = (np.arange(ny) - (ny - 1) / 2) * dx
    X, Y = np.meshgrid(x, y)
    c = 1500 + 40 * np.exp(-((X - 5e-3) ** 2 + Y ** 2) / (2 * (12e-3) ** 2))
    sols = {}
    for precision in ("c64-refined", "tf32-refined"):
        s = HelmholtzSolver(x, y, c, None, 0.8e6, -1, 10.0, 16 * dx, dict(backend="gpu", stencil_bounds=(1400, 1700)),
                            precision=precision, refine_tol=1e-9, max_sources=400)
        out = {}
        for adjoint, S in ((False, 400), (True, 150)):
            r = np.zeros((ny, nx, S), np.complex64)
            g = np.random.default_rng(11 + S)
            r[1:-1, 1:-1] = (g.standard_normal((ny - 2, nx - 2, S)) + 1j * g.standard_normal((ny - 2, nx - 2, S)))
            out[adjoint] = to_np(s.solve(r, adjoint=adjoint))
            st = s.stats()
            assert st["error_estimate"] <= 1e-9, (precision, adjoint, st)
        sols[precision] = out
        s.close()
    for adjoint in (False, True):
        a = sols["tf32-refined"][adjoint][1:-1, 1:-1]
        b = sols["c64-refined"][adjoint][1:-1, 1:-1]
        assert rel(a, b) < 1e-7, adjoint


@pytest.mark.parametrize("ny,nx,S,pml_cells", [(300, 340, 300, 16), (130, 9, 20, 3)])
def test_chunked_sweeps_match_sequential(ny, nx, S, pml_cells):
    """The column-chunked TF32 sweeps (chunks solved concurrently, joined by
    their composed propagators) apply the same block-LU operator as the
    sequential TF32 sweeps: refined to 1e-9 both give the same fields, and
    the chunked sweep needs at most one correction more.  Grids: 26 chunks
    with two source tiles (256 + 44), and 4 chunks on a narrow grid."""
    from waveforminversionust_b200.solver import HelmholtzSolver
    dx = 0.3e-3
    x = (np.arange(nx) - (nx - 1) / 2) * dx
    y = (np.arange(ny) - (ny - 1) / 2) * dx
    X, Y = np.meshgrid(x, y)
    c = 1500 + 40 * np.exp(-((X - 2e-3) ** 2 + Y ** 2) / (2 * (8e-3) ** 2))
    sols, iters = {}, {}
    for method in ("default", "sequential"):
        s = HelmholtzSolver(x, y, c, None, 0.8e6, -1, 10.0, pml_cells * dx,
                            dict(backend="gpu", stencil_bounds=(1400, 1700)), precision="tf32-refined",
                            refine_tol=1e-9, max_sources=S, sweep_method=method,
                            correction_precision="same")
        for adjoint in (False, True):
            r = np.zeros((ny, nx, S), np.complex64)
            g = np.random.default_rng(5 + adjoint)
            r[1:-1, 1:-1] = g.standard_normal((ny - 2, nx - 2, S)) + 1j * g.standard_normal((ny - 2, nx - 2, S))
            sols[method, adjoint] = to_np(s.solve(r, adjoint=adjoint))
            st = s.stats()
            assert st["error_estimate"] <= 1e-9, (method, adjoint, st)
            iters[method, adjoint] = st["refine_iters"]
        s.close()
    for adjoint in (False, True):
        a = sols["default", adjoint][1:-1, 1:-1]
        b = sols["sequential", adjoint][1:-1, 1:-1]
        assert rel(a, b) < 1e-7, adjoint
        assert iters["default", adjoint] <= iters["sequential", adjoint] + 1, iters


def test_bf16_correction_sweeps_match_tf32_corrections():
    """The TF32 profile's correction solves on BF16 operands (pages and chunk
    propagators) reach the same fields as TF32 corrections once refined to
    1e-9, and at the default 1e-5 target need at most one more correction."""
    from waveforminversionust_b200.solver import HelmholtzSolver
    ny, nx, S = 300, 340, 200
    dx = 0.3e-3
    x = (np.arange(nx) - (nx - 1) / 2) * dx
    y = (np.arange(ny) - (ny - 1) / 2) * dx
    X, Y = np.meshgrid(x, y)
    c = 1500 + 40 * np.exp(-((X - 2e-3) ** 2 + Y ** 2) / (2 * (8e-3) ** 2))
    g = np.random.default_rng(9)
    r = np.zeros((ny, nx, S), np.complex64)
    r[1:-1, 1:-1] = g.standard_normal((ny - 2, nx - 2, S)) + 1j * g.standard_normal((ny - 2, nx - 2, S))
    sols, iters = {}, {}
    for corr in ("default", "same"):
        for tol in (1e-9, 1e-5):
            s = HelmholtzSolver(x, y, c, None, 0.8e6, -1, 10.0, 16 * dx, dict(backend="gpu", stencil_bounds=(1400, 1700)),
                                precision="tf32-refined", refine_tol=tol, max_sources=S, correction_precision=corr)
            for adjoint in (False, True):
                sols[corr, tol, adjoint] = to_np(s.solve(r, adjoint=adjoint))
                st = s.stats()
                assert st["error_estimate"] <= tol, (corr, tol, adjoint, st)
                iters[corr, tol, adjoint] = st["refine_iters"]
            s.close()
    for adjoint in (False, True):
        assert rel(sols["default", 1e-9, adjoint][1:-1, 1:-1], sols["same", 1e-9, adjoint][1:-1, 1:-1]) < 1e-7
        assert iters["default", 1e-5, adjoint] <= iters["same", 1e-5, adjoint] + 1, iters


def test_single_correction_returns_the_corrected_field():
    """With a loose target the refinement stops after one correction; the
    returned field is then the corrected iterate (the first correction reads
    the solve's c64 field and writes only the FP64 iterate, whose c64 copy is
    returned), not the uncorrected solve: its error against a 1e-9 solution is
    about the estimate, a hundredth of the correction itself."""
    from waveforminversionust_b200.solver import HelmholtzSolver
    ny, nx, S = 130, 150, 16
    dx = 0.3e-3
    x = (np.arange(nx) - (nx - 1) / 2) * dx
    y = (np.arange(ny) - (ny - 1) / 2) * dx
    X, Y = np.meshgrid(x, y)
    c = 1500 + 40 * np.exp(-((X - 2e-3) ** 2 + Y ** 2) / (2 * (8e-3) ** 2))
    g = np.random.default_rng(11)
    r = np.zeros((ny, nx, S), np.complex64)
    r[1:-1, 1:-1] = g.standard_normal((ny - 2, nx - 2, S)) + 1j * g.standard_normal((ny - 2, nx - 2, S))
    out = {}
    for tol in (1e-9, 3e-2):
        s = HelmholtzSolver(x, y, c, None, 0.8e6, -1, 10.0, 16 * dx, dict(backend="gpu", stencil_bounds=(1400, 1700)),
                            precision="tf32-refined", refine_tol=tol, max_sources=S)
        for adjoint in (False, True):
            out[tol, adjoint] = (to_np(s.solve(r, adjoint=adjoint)), s.stats())
        s.close()
    for adjoint in (False, True):
        u1, st = out[3e-2, adjoint]
        assert st["refine_iters"] == 1, st
        err = rel(u1[1:-1, 1:-1], out[1e-9, adjoint][0][1:-1, 1:-1])
        assert err <= 10 * st["error_estimate"] + 1e-6, (adjoint, err, st)


def test_newton_schulz_factor_agrees_with_gauss_jordan():
    """The TF32 profile's Schur inverses (Newton-Schulz iterations on the
    tensor cores, Gauss-Jordan on the pages where the previous inverse is no
    start) agree with the complex-single Gauss-Jordan pages to TF32 accuracy,
    on a textured medium where the iteration needs several steps."""
    from waveforminversionust_b200.solver import HelmholtzSolver
    ny = nx = 330
    dx = 0.3e-3
    x = (np.arange(nx) - (nx - 1) / 2) * dx
    y = (np.arange(ny) - (ny - 1) / 2) * dx
    X, Y = np.meshgrid(x, y)
    rng = np.random.default_rng(5)
    c = 1500 + 60 * np.exp(-((X - 4e-3) ** 2 + Y ** 2) / (2 * (15e-3) ** 2)) + 5 * rng.standard_normal(X.shape)
    opts = dict(backend="gpu", stencil_bounds=(1400, 1700))
    ref = HelmholtzSolver(x, y, c, None, 0.8e6, -1, 10.0, 16 * dx, opts, precision="c64", max_sources=4)
    tc = HelmholtzSolver(x, y, c, None, 0.8e6, -1, 10.0, 16 * dx, opts, precision="tf32-refined", max_sources=4)
    a = to_np(ref.block("invT"))
    b = to_np(tc.block("invT"))
    st = tc.factor_stats()
    assert st["newton_schulz_pages"] + st["gauss_jordan_pages"] == nx, st
    assert st["newton_schulz_pages"] >= nx // 2, st
    assert st["gemms"] >= 2 * st["newton_schulz_pages"] - nx, st
    # the Dirichlet columns' pages are the identity, written in closed form
    for j in (0, nx - 1):
        assert np.array_equal(b[1:-1, 1:-1, j], np.eye(ny - 2)), j
    per_page = np.linalg.norm((b - a).reshape(-1, nx), axis=0) / np.linalg.norm(a.reshape(-1, nx), axis=0)
    assert per_page.max() < 5e-3, (per_page.argmax(), per_page.max())
    assert rel(b, a) < 2e-3
    ref.close()
    tc.close()


def test_newton_schulz_cluster_kernel_matches_classic_kernel(monkeypatch):
    """The Newton-Schulz kernel launched as clusters (the K slices of a tile
    sum their split-K partials through distributed shared memory) gives the
    same Schur inverses, bit for bit, as the kernel whose partials go through
    L2 (same K split, same summation order), with the same page decisions,
    on a textured grid where pages take the cubic, quadratic and Gauss-Jordan
    routes."""
    from waveforminversionust_b200.solver import HelmholtzSolver
    ny = nx = 482                     # 480 interior rows: 8 x 5 tiles, K split 3 either way
    dx = 0.3e-3
    x = (np.arange(nx) - (nx - 1) / 2) * dx
    y = (np.arange(ny) - (ny - 1) / 2) * dx
    X, Y = np.meshgrid(x, y)
    rng = np.random.default_rng(11)
    c = 1500 + 60 * np.exp(-((X - 4e-3) ** 2 + Y ** 2) / (2 * (20e-3) ** 2)) + 5 * rng.standard_normal(X.shape)
    opts = dict(backend="gpu", stencil_bounds=(1400, 1700))
    monkeypatch.setenv("WUST_NS_CLUSTER", "0")
    classic = HelmholtzSolver(x, y, c, None, 0.8e6, -1, 10.0, 16 * dx, opts, precision="tf32-refined",
                              max_sources=4)
    monkeypatch.delenv("WUST_NS_CLUSTER")
    clustered = HelmholtzSolver(x, y, c, None, 0.8e6, -1, 10.0, 16 * dx, opts, precision="tf32-refined",
                                max_sources=4)
    ia, ib = classic.factor_info(), clustered.factor_info()
    assert ia == {"k_slices": 3, "cluster": 0}, ia
    assert ib == {"k_slices": 3, "cluster": 1}, ib
    sa, sb = classic.factor_stats(), clustered.factor_stats()
    assert sa == sb, (sa, sb)
    assert sa["gemms"] > 2 * sa["newton_schulz_pages"], sa      # cubic / repeated updates were taken
    a = to_np(classic.block("invT"))
    b = to_np(clustered.block("invT"))
    assert np.array_equal(np.ascontiguousarray(a).view(np.uint32), np.ascontiguousarray(b).view(np.uint32))
    classic.close()
    clustered.close()


def test_mass_apply_matches_oracle(small):
    p, ref = small
    s = make_gpu_solver(p, p.c_true, p.frequencies_hz[0])
    rng = np.random.default_rng(2)
    ny, nx = p.shape
    v = (rng.standard_normal((ny, nx, 3)) + 1j * rng.standard_normal((ny, nx, 3))).astype(np.complex64)
    for adjoint in (False, True):
        got = to_np(s.massApply(v, adjoint))
        want = ref.mass_apply(v.astype(np.complex128), adjoint)
        assert rel(got, want) < 1e-6
    s.close()


def _gpu_obs(o_obs):
    from waveforminversionust_b200.objective import Observations
    return Observations(o_obs.x_m, o_obs.y_m, o_obs.tx_index, o_obs.rx_index, o_obs.frequencies_hz, o_obs.Y,
                        o_obs.mask)


@pytest.mark.parametrize("precision,tol_loss,tol_grad", [("c64", 1e-3, 1e-2), ("c64-refined", 1e-7, 1e-5),
                                                        ("tf32-refined", 1e-7, 1e-5)])
def test_oracle_matches_reference_fixture(ref_fixture, precision, tol_loss, tol_grad):
    """wust_oracle on the 31x31 fixture of test_runtime.m: loss and gradient."""
    from oracle import helmholtz_fp64 as o
    from waveforminversionust_b200.objective import POOL, default_config, wust_oracle
    fx = ref_fixture
    loss_ref, grad_ref, _ = o.wust_oracle(fx["initial"], fx["obs"], 0, fx["cfg"])
    cfg = default_config(pml_m=.004, pml_strength=10, source_batch_size=2, precision=precision, refine_tol=1e-10)
    obs = _gpu_obs(fx["obs"])
    loss, grad = wust_oracle(fx["initial"], obs, 0, cfg)
    assert abs(loss - loss_ref) / loss_ref < tol_loss
    assert rel(grad, grad_ref) < tol_grad
    loss_only = wust_oracle(fx["initial"], obs, 0, cfg, nargout=1)
    assert abs(loss_only - loss) <= 1e-6 * loss          # test_runtime.m:53-55
    POOL.clear()


def test_gradient_finite_difference_gpu(ref_fixture):
    """Central FD vs adjoint gradient (test_runtime.m:45-56,192-201); refined
    profile meets the FP64 tolerance 1e-4 instead of the c64 0.03."""
    from waveforminversionust_b200.objective import POOL, default_config, wust_oracle
    fx = ref_fixture
    obs = _gpu_obs(fx["obs"])
    cfg = default_config(pml_m=.004, pml_strength=10, source_batch_size=2, precision="c64-refined",
                         refine_tol=1e-10)
    init, direction, step = fx["initial"], fx["direction"], 1e-3
    _, g = wust_oracle(init, obs, 0, cfg)
    lp = wust_oracle(1 / (1 / init + step * direction), obs, 0, cfg, nargout=1)
    lm = wust_oracle(1 / (1 / init - step * direction), obs, 0, cfg, nargout=1)
    fd = (lp - lm) / (2 * step)
    adj = float(np.sum(g * direction))
    assert abs(fd - adj) / max(abs(fd), abs(adj)) < 1e-4
    # c64 profile with the reference's GPU step and tolerance
    cfg64 = default_config(pml_m=.004, pml_strength=10, source_batch_size=2, precision="c64")
    _, g = wust_oracle(init, obs, 0, cfg64)
    step = .1
    lp = wust_oracle(1 / (1 / init + step * direction), obs, 0, cfg64, nargout=1)
    lm = wust_oracle(1 / (1 / init - step * direction), obs, 0, cfg64, nargout=1)
    fd = (lp - lm) / (2 * step)
    adj = float(np.sum(g * direction))
    assert abs(fd - adj) / max(abs(fd), abs(adj)) < 0.03
    POOL.clear()


def test_batch_invariance(ref_fixture):
    """source_batch_size 2 vs 3 (test_runtime.m:57-61)."""
    from waveforminversionust_b200.objective import POOL, default_config, wust_oracle
    fx = ref_fixture
    obs = _gpu_obs(fx["obs"])
    l2, g2 = wust_oracle(fx["initial"], obs, 0, default_config(pml_m=.004, source_batch_size=2))
    l3, g3 = wust_oracle(fx["initial"], obs, 0, default_config(pml_m=.004, source_batch_size=3))
    assert abs(l3 - l2) / l2 < 1e-4
    assert rel(g3, g2) < 1e-4
    POOL.clear()


def test_curvature_matches_oracle(ref_fixture):
    from oracle import helmholtz_fp64 as o
    from waveforminversionust_b200.objective import POOL, default_config, directional_curvature, wust_oracle
    fx = ref_fixture
    _, _, state_ref = o.wust_oracle(fx["initial"], fx["obs"], 0, fx["cfg"], retain_state=True)
    k_ref = o.directional_curvature(state_ref, fx["direction"], fx["obs"].rx_index, fx["obs"].mask[:, :, 0])
    obs = _gpu_obs(fx["obs"])
    cfg = default_config(pml_m=.004, source_batch_size=2, precision="c64-refined")
    _, _, state = wust_oracle(fx["initial"], obs, 0, cfg, nargout=3)
    k = directional_curvature(state, fx["direction"])
    assert abs(k - k_ref) / k_ref < 1e-6
    POOL.clear()


def test_config1_gradient_parity():
    """Config-1 sized gradient (224^2 incl. PML, 32 TX, 128 RX) vs the FP64 sparse LU."""
    from oracle import helmholtz_fp64 as o
    from waveforminversionust_b200 import synthetic
    from waveforminversionust_b200.objective import POOL, Observations, default_config, wust_oracle
    p = synthetic.config1(seed=1)
    cfg_o = o.OracleConfig(pml_m=p.pml_m)
    dummy = o.Observations(p.x_m, p.y_m, p.tx_index, p.rx_index, p.frequencies_hz,
                           np.zeros((32, 128, 1)), np.ones((32, 128, 1), bool))
    true_solver = o.make_solver(p.c_true, dummy, 0, cfg_o)
    ny, nx = p.shape
    u = true_solver.solve(o.point_sources(p.tx_index, range(32), ny, nx))
    Yobs = u.reshape(-1, 32, order="F")[p.rx_index - 1, :].T[:, :, None]
    o_obs = o.Observations(p.x_m, p.y_m, p.tx_index, p.rx_index, p.frequencies_hz, Yobs, np.ones((32, 128, 1), bool))
    loss_ref, grad_ref, _ = o.wust_oracle(p.c_init, o_obs, 0, cfg_o)
    obs = Observations(p.x_m, p.y_m, p.tx_index, p.rx_index, p.frequencies_hz, Yobs, np.ones((32, 128, 1), bool))
    # Refined profiles stop at an estimated forward error of 1e-5 (the pressure
    # tolerance); the TF32 sweeps contract less per correction than the
    # complex-single ones, so their misfit is held to that 1e-5 bound.
    for precision, tl, tg in (("c64", 1e-3, 1e-2), ("c64-refined", 1e-6, 1e-4), ("tf32-refined", 1e-5, 1e-4),
                              ("bf16-refined", 1e-5, 1e-4)):
        loss, grad = wust_oracle(p.c_init, obs, 0, default_config(pml_m=p.pml_m, precision=precision))
        assert abs(loss - loss_ref) / loss_ref < tl, precision
        assert rel(grad, grad_ref) < tg, precision
        POOL.clear()


def test_invalid_inputs_raise_reference_ids(small):
    import torch
    from waveforminversionust_b200._lib import WustError
    from waveforminversionust_b200.solver import HelmholtzSolver, applyBlockLU
    p, ref = small
    for bad in (dict(stencil_bounds=(1400, 1700)), dict(backend="gpu"), dict(backend="gpu", stencil_bounds=None),
                dict(backend="gpu", stencil_bounds=(1500,))):
        with pytest.raises(WustError) as e:
            HelmholtzSolver(p.x_m, p.y_m, p.c_true, None, 3e5, -1, 10, p.pml_m, bad)
        assert e.value.identifier == "WUST:InvalidInput"
    c = ref.coefs
    # inconsistent shapes -> InvalidInput before any device access
    with pytest.raises(WustError) as e:
        applyBlockLU(torch.zeros((2, 2, 2, 2), dtype=torch.complex64), c["Ld"], c["Ll"], c["Lu"], c["Ud"], c["Ul"],
                     c["Uu"], torch.zeros((2, 2, 2), dtype=torch.complex64), False)
    assert e.value.identifier == "WUST:InvalidInput"


def test_degenerate_data_is_numerical_failure(ref_fixture):
    """All receivers masked -> unusable source-scale denominator (wust_oracle.m:55-57)."""
    from waveforminversionust_b200._lib import WustError
    from waveforminversionust_b200.objective import POOL, Observations, default_config, wust_oracle
    fx = ref_fixture
    o = fx["obs"]
    mask = np.ones_like(o.mask)
    mask[0, :, 0] = False
    obs = Observations(o.x_m, o.y_m, o.tx_index, o.rx_index, o.frequencies_hz, o.Y, mask)
    with pytest.raises(WustError) as e:
        wust_oracle(fx["initial"], obs, 0, default_config(pml_m=.004))
    assert e.value.identifier == "WUST:NumericalFailure"
    POOL.clear()


def test_bounded_device_wait_times_out():
    """A grid barrier that can never fill must give up within its budget and
    leave the context usable (no trap, no hang)."""
    import ctypes as C
    import torch
    from waveforminversionust_b200 import _lib
    lib = _lib.load()
    site = C.c_int()
    rc = lib.wust_selftest_barrier_timeout(50, C.byref(site))
    assert rc == 11 and site.value == 77
    x = torch.ones(16, device="cuda")
    assert float((x * 2).sum()) == 32.0
