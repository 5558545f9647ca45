"""Parity at the benchmark's own configuration against the FP64 sparse LU.

The timed workload is a 552 x 552 grid (512^2 interior + 20-cell PML, dx
0.25 mm), 256 transmitters and 256 receivers on a 55 mm ring, 1.2 MHz, on
the seeded breast-like phantom.  These tests run the same solver objects the
benchmark times (256-source batches through the column-chunked tensor-core
sweeps and the Newton-Schulz factorization for the TF32 profile) and compare
them with SciPy's complex128 sparse LU, the stand-in for the reference's CPU
``decomposition(H,'lu')`` (Runtime/solver/HelmholtzSolver.m:114-143), on two
media: the homogeneous starting model of the first NCG iteration and the
textured phantom itself.

Tolerances are the targets of the path: pressure within 1e-5 relative L2
(forward fields, and adjoint fields on the interior: the block solver leaves
its own values on the Dirichlet ring, which M^T zeroes before use,
HelmholtzSolver.m:211-219), misfit within 1e-5 and gradient within 1e-4.
Pressure is checked on 8 transmitters spread over the ring, sampled from
the 256-source solve; the gradient on every 16th transmitter (16 of them),
through the same kernels.
"""
import numpy as np
import pytest
import torch

from conftest import gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]

FREQ = 1.2e6
SAMPLE = [0, 37, 73, 110, 146, 183, 219, 255]
GRAD_TX = list(range(0, 256, 16))
MODELS = ("homogeneous", "textured")
PROFILES = ("tf32-refined", "c64-refined", "bf16-refined")


def rel(a, b):
    return float(np.linalg.norm((np.asarray(a) - np.asarray(b)).ravel()) / np.linalg.norm(np.asarray(b).ravel()))


@pytest.fixture(scope="module")
def headline():
    """The config-2 problem and a lazily built FP64 sparse-LU solver per medium."""
    from oracle import helmholtz_fp64 as o
    from waveforminversionust_b200 import synthetic
    p = synthetic.config2(seed=0, freqs=[FREQ])
    media = dict(homogeneous=p.c_init, textured=p.c_true)
    solvers = {}

    def fp64(name):
        if name not in solvers:
            solvers[name] = o.HelmholtzSolverFP64(p.x_m, p.y_m, media[name], np.zeros(p.shape), FREQ, -1, 10.0,
                                                  p.pml_m, dict(backend="cpu", stencil_bounds=(1400, 1700)))
        return solvers[name]

    return p, media, fp64


def _point_sources_device(p):
    ny, nx = p.shape
    n = p.tx_index.size
    src = torch.zeros((n, nx, ny), dtype=torch.complex64, device="cuda")
    src.view(n, -1)[torch.arange(n, device="cuda"), torch.as_tensor(p.tx_index - 1, device="cuda")] = 1
    return src.permute(2, 1, 0)


def _receiver_sources(p, seed):
    """Adjoint right-hand sides like the oracle's: residuals scattered at the receivers."""
    ny, nx = p.shape
    n = p.tx_index.size
    rng = np.random.default_rng(seed)
    r = np.zeros((ny * nx, n), np.complex64)
    r[p.rx_index - 1, :] = rng.standard_normal((p.rx_index.size, n)) + 1j * rng.standard_normal((p.rx_index.size, n))
    return r.reshape(ny, nx, n, order="F")


@pytest.mark.parametrize("precision", PROFILES)
@pytest.mark.parametrize("model", MODELS)
def test_headline_pressure_matches_fp64_sparse_lu(headline, model, precision):
    from oracle import helmholtz_fp64 as o
    from waveforminversionust_b200.solver import HelmholtzSolver
    p, media, fp64 = headline
    ny, nx = p.shape
    s = HelmholtzSolver(p.x_m, p.y_m, media[model], None, FREQ, -1, 10.0, p.pml_m,
                        dict(backend="gpu", stencil_bounds=(1400, 1700)), precision=precision, max_sources=256)
    ref = fp64(model)
    u = s.solve(_point_sources_device(p))[:, :, SAMPLE].cpu().numpy()
    st_f = s.stats()
    want = ref.solve(o.point_sources(p.tx_index, SAMPLE, ny, nx))
    per_tx = [rel(u[:, :, k], want[:, :, k]) for k in range(len(SAMPLE))]
    assert rel(u, want) <= 1e-5, (model, precision, per_tx, st_f)
    assert max(per_tx) <= 2e-5, (model, precision, per_tx, st_f)

    r = _receiver_sources(p, seed=7)
    lam = s.solve(r, adjoint=True)[:, :, SAMPLE].cpu().numpy()
    st_a = s.stats()
    lam_ref = ref.solve(r[:, :, SAMPLE].astype(np.complex128), adjoint=True)
    per_tx = [rel(lam[1:-1, 1:-1, k], lam_ref[1:-1, 1:-1, k]) for k in range(len(SAMPLE))]
    assert rel(lam[1:-1, 1:-1], lam_ref[1:-1, 1:-1]) <= 1e-5, (model, precision, per_tx, st_a)
    assert max(per_tx) <= 2e-5, (model, precision, per_tx, st_a)
    s.close()


@pytest.mark.parametrize("model", MODELS)
def test_headline_misfit_and_gradient_match_fp64_oracle(headline, model):
    """wust_oracle at the benchmark grid and frequency with 16 transmitters:
    observations are FP64 solves on the other medium, so the residual is
    large at both evaluation points."""
    from oracle import helmholtz_fp64 as o
    from waveforminversionust_b200.objective import POOL, Observations, default_config, wust_oracle
    p, media, fp64 = headline
    ny, nx = p.shape
    other = "textured" if model == "homogeneous" else "homogeneous"
    tx = p.tx_index[GRAD_TX]
    n_tx, n_rx = tx.size, p.rx_index.size
    u_obs = fp64(other).solve(o.point_sources(tx, range(n_tx), ny, nx))
    Y = u_obs.reshape(ny * nx, n_tx, order="F")[p.rx_index - 1, :].T[:, :, None]
    mask = np.ones((n_tx, n_rx, 1), bool)
    o_obs = o.Observations(p.x_m, p.y_m, tx, p.rx_index, np.array([FREQ]), Y, mask)
    cfg_o = o.OracleConfig(pml_m=p.pml_m, source_batch_size=n_tx)
    loss_ref, grad_ref, _ = o.wust_oracle(media[model], o_obs, 0, cfg_o, solver=fp64(model))
    obs = Observations(p.x_m, p.y_m, tx, p.rx_index, np.array([FREQ]), Y, mask)
    for precision in PROFILES:
        loss, grad = wust_oracle(media[model], obs, 0,
                                 default_config(pml_m=p.pml_m, precision=precision, source_batch_size=n_tx))
        e_loss = abs(loss - loss_ref) / loss_ref
        e_grad = rel(grad, grad_ref)
        assert e_loss <= 1e-5, (model, precision, e_loss)
        assert e_grad <= 1e-4, (model, precision, e_grad)
        POOL.clear()
