"""The MATLAB boundary, run without MATLAB through the MEX runtime stand-in.

Two kinds of MEX code are loaded into the stand-in (oracle/mexshim):

* the reference's own kernels, Runtime/solver/decompBlockLU.cu and
  applyBlockLU.cu, compiled unchanged (pivoted cuSOLVER LU per Schur page,
  cuBLAS Cgemm3m sweeps) -- they pin the oracle's block-LU restatement and
  are the parity target of this repository's complex-single block LU;
* this repository's gateways (waveforminversionust_b200/mex/*.c), built
  against the same stand-in, fed the same mxArrays.

CPU tests cover argument handling and error identifiers (they fail before
any device work); GPU tests compare outputs.
"""
import numpy as np
import pytest

from conftest import gpu_available

NAMES = ("Ld", "Ll", "Lu", "Dd", "Dl", "Du", "Ud", "Ul", "Uu")


@pytest.fixture(scope="module")
def mex(tmp_path_factory):
    from oracle.mexshim import driver
    rt = driver.runtime()
    out = str(tmp_path_factory.mktemp("mex"))
    ours = {n: driver.gateway(n, out) for n in ("decompBlockLU", "applyBlockLU", "wust_solver")}
    ref = driver.reference_kernels() if driver.reference_available() else {}
    return rt, ours, ref


def _raises(rt, fn, nlhs, *args):
    from oracle.mexshim.driver import MexError
    with pytest.raises(MexError) as e:
        rt.call(fn, nlhs, *args)
    return e.value.identifier


def test_gateways_reject_bad_arguments_with_reference_identifiers(mex):
    rt, ours, ref = mex
    host = [rt.host(np.zeros((4, 3), np.complex64)) for _ in range(9)]
    for impl in [ours] + ([ref] if ref else []):
        assert _raises(rt, impl["decompBlockLU"], 1, *host[:8]) == "WUST:InvalidInput"     # 8 inputs
        assert _raises(rt, impl["decompBlockLU"], 3, *host) == "WUST:InvalidOutput"       # 3 outputs
        assert _raises(rt, impl["decompBlockLU"], 1, *host) == "WUST:InvalidInput"        # host, not gpuArray
        assert _raises(rt, impl["applyBlockLU"], 2, *host) == "WUST:InvalidOutput"
        assert _raises(rt, impl["applyBlockLU"], 1, *host[:8], rt.host(np.ones(2))) == "WUST:InvalidInput"
    ws = ours["wust_solver"]
    assert _raises(rt, ws, 0, "nonsense", np.uint64(1)) == "WUST:InvalidInput"
    assert _raises(rt, ws, 0, rt.string("info"), rt.host(np.array([[7]], np.uint64))) == "WUST:InvalidInput"
    x = np.arange(8) * 1e-3
    vel = np.full((8, 8), 1500.0)
    for opts in (dict(backend="gpu"), dict(stencil_bounds=np.array([1400.0, 1700.0])),
                 dict(backend="gpu", stencil_bounds=np.array([1700.0, 1400.0])),
                 dict(backend="cpu", stencil_bounds=np.array([1400.0, 1700.0])),
                 dict(backend="gpu", stencil_bounds=np.array([1400.0, 1700.0]), precision="fp8")):
        ident = _raises(rt, ws, 1, "create", x, x, vel, np.zeros((0, 0)), 3e5, -1.0, 10.0, 2e-3, rt.struct(opts))
        assert ident == "WUST:InvalidInput", opts


gpu = pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")


def _blocks(p, c, f):
    from oracle import helmholtz_fp64 as o
    s = o.HelmholtzSolverFP64(p.x_m, p.y_m, c, np.zeros(p.shape), f, -1, 10.0, p.pml_m,
                              dict(backend="cpu", stencil_bounds=(1400, 1700)), factor=False)
    return s


def _gpu_colmajor(rt, a):
    import torch
    a = np.asarray(a, np.complex64)
    t = torch.as_tensor(np.ascontiguousarray(a.T), device="cuda")       # reversed dims, contiguous
    return rt.gpu(t.permute(*reversed(range(t.dim()))), dims=a.shape)


def rel(a, b):
    return float(np.linalg.norm((np.asarray(a) - np.asarray(b)).ravel()) / np.linalg.norm(np.asarray(b).ravel()))


@pytest.mark.gpu
@gpu
@pytest.mark.parametrize("case", ["small", "config1"])
def test_block_lu_matches_the_reference_kernels(mex, case):
    """decompBlockLU / applyBlockLU: the reference's own kernels against the
    FP64 restatement (the oracle's pin) and this repository's gateways
    against the reference's kernels, on the same gpuArrays."""
    from oracle import helmholtz_fp64 as o
    from waveforminversionust_b200 import synthetic
    rt, ours, ref = mex
    if not ref:
        pytest.skip("reference MEX kernels not built (needs the reference sources at build time)")
    p = synthetic.small(seed=4) if case == "small" else synthetic.config1(seed=2)
    f = float(p.frequencies_hz[0])
    s = _blocks(p, p.c_true, f)
    blocks = [_gpu_colmajor(rt, s.coefs[n]) for n in NAMES]
    want = o.block_lu_factor(s.coefs)
    (inv_ref, info) = rt.call(ref["decompBlockLU"], 2, *blocks)
    (inv_ours, info_ours) = rt.call(ours["decompBlockLU"], 2, *blocks)
    a, b = inv_ref.numpy(), inv_ours.numpy()
    assert a.shape == b.shape == want.shape
    e_ref, e_ours = rel(a, want), rel(b, want)
    assert e_ref < 1e-4, e_ref                  # the oracle's recursion agrees with the reference's kernels
    assert e_ours < max(2 * e_ref, 2e-5), (e_ours, e_ref)
    assert rel(b, a) < 1e-4
    assert info.field("block_count").scalar() == info_ours.field("block_count").scalar() == p.shape[1]
    ny, nx = p.shape
    rng = np.random.default_rng(1)
    src = np.zeros((ny, nx, 6), np.complex64)
    src[1:-1, 1:-1] = rng.standard_normal((ny - 2, nx - 2, 6)) + 1j * rng.standard_normal((ny - 2, nx - 2, 6))
    lu = [blocks[i] for i in (0, 1, 2, 6, 7, 8)]
    for adjoint in (False, True):
        (u_ref,) = rt.call(ref["applyBlockLU"], 1, _gpu_colmajor(rt, src), *lu, inv_ref, rt.logical(adjoint))
        (u_ours,) = rt.call(ours["applyBlockLU"], 1, _gpu_colmajor(rt, src), *lu, inv_ours, rt.logical(adjoint))
        u_want = o.block_lu_apply(src.astype(np.complex128), s.coefs, want, adjoint)
        e_ref, e_ours = rel(u_ref.numpy(), u_want), rel(u_ours.numpy(), u_want)
        assert e_ref < 1e-4, (adjoint, e_ref)
        assert e_ours < max(2 * e_ref, 5e-5), (adjoint, e_ours, e_ref)


@pytest.mark.gpu
@gpu
def test_singular_schur_block_is_reported_like_the_reference(mex):
    """A host-built operator whose first Schur block is zero: both the
    reference's kernels (cuSOLVER info > 0) and this repository's
    factorization report WUST:SingularSchurBlock, and the device keeps
    answering."""
    import torch
    rt, ours, ref = mex
    ny, nx = 31, 6
    rng = np.random.default_rng(3)
    shapes = dict(Ld=(ny, nx - 1), Ll=(ny - 1, nx - 1), Lu=(ny - 1, nx - 1), Dd=(ny, nx), Dl=(ny - 1, nx),
                  Du=(ny - 1, nx), Ud=(ny, nx - 1), Ul=(ny - 1, nx - 1), Uu=(ny - 1, nx - 1))
    coefs = {n: (0.1 * rng.standard_normal(sh)).astype(np.complex64) for n, sh in shapes.items()}
    coefs["Dd"][:, 1:] += 4
    for n in ("Dd", "Dl", "Du"):
        coefs[n][:, 0] = 0                      # T_1 = D_1 = 0: singular at its first pivot
    blocks = [_gpu_colmajor(rt, coefs[n]) for n in NAMES]
    for impl in [ours] + ([ref] if ref else []):
        assert _raises(rt, impl["decompBlockLU"], 1, *blocks) == "WUST:SingularSchurBlock"
    x = torch.ones(8, device="cuda")
    assert float((2 * x).sum()) == 16.0


@pytest.mark.gpu
@gpu
@pytest.mark.parametrize("precision", ["c64", "tf32-refined"])
def test_wust_solver_gateway_matches_fp64_oracle(mex, precision):
    """The whole-object gateway: create with a precision profile, solve,
    massApply, the oracle's misfit and gradient, curvature, info, destroy."""
    from oracle import helmholtz_fp64 as o
    from waveforminversionust_b200 import synthetic
    rt, ours, _ = mex
    ws = ours["wust_solver"]
    p = synthetic.small(seed=6)
    ny, nx = p.shape
    f = float(p.frequencies_hz[0])
    opts = rt.struct(dict(backend="gpu", stencil_bounds=np.array([1400.0, 1700.0]), precision=precision,
                          refine_tol=1e-6, max_sources=16.0))
    (h,) = rt.call(ws, 1, "create", p.x_m, p.y_m, p.c_init, np.zeros((0, 0)), f, -1.0, 10.0, p.pml_m, opts)
    try:
        fp = _blocks(p, p.c_init, f)
        fp.lu = o.spla.splu(fp.H)
        n_tx = p.tx_index.size
        src = o.point_sources(p.tx_index, range(n_tx), ny, nx)
        u, virt = rt.call(ws, 2, "solve", h, _gpu_colmajor(rt, src), rt.logical(False))
        want = fp.solve(src)
        tol = 1e-3 if precision == "c64" else 2e-6
        assert rel(u.numpy(), want) < tol
        assert rel(virt.numpy(), want * fp.virtual_source_multiplier[:, :, None]) < tol
        (m,) = rt.call(ws, 1, "massApply", h, u, rt.logical(True))
        assert rel(m.numpy(), fp.mass_apply(u.numpy().astype(np.complex128), True)) < 1e-6
        info = rt.call(ws, 1, "info", h)[0]
        assert abs(info.field("massD").scalar() - fp.d) < 1e-12
        # the oracle on observations simulated on the true medium
        tru = _blocks(p, p.c_true, f)
        tru.lu = o.spla.splu(tru.H)
        Y = tru.solve(src).reshape(ny * nx, n_tx, order="F")[p.rx_index - 1, :].T
        mask = np.ones(Y.shape, bool)
        obs = o.Observations(p.x_m, p.y_m, p.tx_index, p.rx_index, [f], Y[:, :, None], mask[:, :, None])
        loss_ref, grad_ref, state = o.wust_oracle(p.c_init, obs, 0, o.OracleConfig(pml_m=p.pml_m), solver=fp,
                                                  retain_state=True)
        loss, grad = rt.call(ws, 2, "oracle", h, p.tx_index.astype(np.float64), p.rx_index.astype(np.float64),
                             rt.host(Y.astype(np.complex64)), rt.host(mask), float(n_tx), rt.logical(True))
        tl, tg = (1e-3, 1e-2) if precision == "c64" else (1e-6, 1e-4)
        assert abs(loss.scalar() - loss_ref) / loss_ref < tl
        assert rel(grad.numpy(), grad_ref) < tg
        direction = np.exp(-((np.arange(ny)[:, None] - ny / 2) ** 2 + (np.arange(nx)[None, :] - nx / 2) ** 2) / 50.0)
        (k,) = rt.call(ws, 1, "curvature", h, direction)
        k_ref = o.directional_curvature(state, direction, p.rx_index, mask)
        assert abs(k.scalar() - k_ref) / k_ref < (1e-2 if precision == "c64" else 1e-5)
        # a new medium on the same grid
        rt.call(ws, 0, "refactor", h, p.c_true, np.zeros((0, 0)), f)
        (u2,) = rt.call(ws, 1, "solve", h, _gpu_colmajor(rt, src), rt.logical(False))
        assert rel(u2.numpy(), tru.solve(src)) < tol
    finally:
        rt.call(ws, 0, "destroy", h)
    assert _raises(rt, ws, 0, "info", h) == "WUST:InvalidInput"        # the handle is gone


@pytest.mark.gpu
@gpu
@pytest.mark.parametrize("dx_mm", [0.40, 0.45])
def test_unpivoted_factor_at_the_stencil_limits(mex, dx_mm):
    """This repository factors each Schur page without pivoting, where the
    reference pivots (cusolverDnCgetrf, decompBlockLU.cu:338-343).  At the
    edge of the operator's range -- 2.6-2.9 points per wavelength at 1.2 MHz
    in 1400 m/s, inclusions at both stencil bounds (1400 and 1700 m/s) and a
    textured background -- the unpivoted pages must be as accurate as the
    reference's pivoted ones against the FP64 recursion, and the refined TF32
    solve must still reach 1e-5 against the FP64 sparse LU."""
    from oracle import helmholtz_fp64 as o
    from waveforminversionust_b200 import synthetic
    from waveforminversionust_b200.solver import HelmholtzSolver
    rt, ours, ref = mex
    if not ref:
        pytest.skip("reference MEX kernels not built (needs the reference sources at build time)")
    n, f = 160, 1.2e6
    dx = dx_mm * 1e-3
    x = synthetic.grid_centres(n, dx)
    X, Y = np.meshgrid(x, x)
    rng = np.random.default_rng(8)
    c = 1500.0 + 8.0 * synthetic._smooth_noise(rng, X.shape, 1.5)
    c[(X - 0.15 * n * dx) ** 2 + Y ** 2 < (0.12 * n * dx) ** 2] = 1400.0
    c[(X + 0.15 * n * dx) ** 2 + (Y - 0.1 * n * dx) ** 2 < (0.1 * n * dx) ** 2] = 1700.0
    c = np.clip(c, 1400.0, 1700.0)
    s = o.HelmholtzSolverFP64(x, x, c, np.zeros(c.shape), f, -1, 10.0, 16 * dx,
                              dict(backend="cpu", stencil_bounds=(1400, 1700)))
    blocks = [_gpu_colmajor(rt, s.coefs[k]) for k in NAMES]
    want = o.block_lu_factor(s.coefs)
    (inv_ref,) = rt.call(ref["decompBlockLU"], 1, *blocks)
    (inv_ours,) = rt.call(ours["decompBlockLU"], 1, *blocks)
    a, b = inv_ref.numpy(), inv_ours.numpy()
    e_ref, e_ours = rel(a, want), rel(b, want)
    page_ref = np.linalg.norm((a - want).reshape(-1, n), axis=0) / np.linalg.norm(want.reshape(-1, n), axis=0)
    page_ours = np.linalg.norm((b - want).reshape(-1, n), axis=0) / np.linalg.norm(want.reshape(-1, n), axis=0)
    assert np.all(np.isfinite(b))
    assert e_ours <= max(2 * e_ref, 2e-5), (e_ours, e_ref)
    assert page_ours.max() <= max(2 * page_ref.max(), 5e-5), (page_ours.max(), page_ref.max())
    tc = HelmholtzSolver(x, x, c, None, f, -1, 10.0, 16 * dx, dict(backend="gpu", stencil_bounds=(1400, 1700)),
                         precision="tf32-refined", max_sources=32)
    tx = rng.choice(np.arange(20, n - 20), size=(32, 2))
    src = np.zeros((n, n, 32), np.complex64)
    src[tx[:, 0], tx[:, 1], np.arange(32)] = 1
    u = tc.solve(src).cpu().numpy()
    st = tc.stats()
    assert rel(u, s.solve(src.astype(np.complex128))) <= 1e-5, st
    tc.close()
