"""Independent inversions sharing one GPU (config 5's batching): problems run
concurrently on SM partitions, each on its own stream with its cooperative
kernels capped, give the gradients they give alone on the whole GPU, and
those agree with the FP64 oracle."""
import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]


def _problems():
    from oracle import helmholtz_fp64 as o
    from waveforminversionust_b200 import synthetic
    from waveforminversionust_b200.batch import BatchProblem
    out, refs = [], []
    for k, (n, n_tx, f) in enumerate([(48, 6, 0.3e6), (64, 8, 0.4e6), (80, 10, 0.35e6), (96, 12, 0.45e6)]):
        p = synthetic.small(seed=10 + k, n_interior=n, n_tx=n_tx, n_elem=2 * n_tx, freqs=(f,))
        ny, nx = p.shape
        n_rx = p.rx_index.size
        dummy = o.Observations(p.x_m, p.y_m, p.tx_index, p.rx_index, [f], np.zeros((n_tx, n_rx, 1)),
                               np.ones((n_tx, n_rx, 1), bool))
        cfg = o.OracleConfig(pml_m=p.pml_m)
        u = o.make_solver(p.c_true, dummy, 0, cfg).solve(o.point_sources(p.tx_index, range(n_tx), ny, nx))
        Y = u.reshape(-1, n_tx, order="F")[p.rx_index - 1, :].T
        mask = np.ones((n_tx, n_rx), bool)
        obs = o.Observations(p.x_m, p.y_m, p.tx_index, p.rx_index, [f], Y[:, :, None], mask[:, :, None])
        loss, grad, _ = o.wust_oracle(p.c_init, obs, 0, cfg)
        out.append(BatchProblem(p.x_m, p.y_m, p.c_init, f, p.pml_m, p.tx_index, p.rx_index, Y, mask,
                                precision="tf32-refined", name=f"small{n}"))
        refs.append((loss, grad))
    return out, refs


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_concurrent_partitions_match_whole_gpu_and_fp64_oracle():
    import torch
    from waveforminversionust_b200.batch import Autotuner, Plan, lpt, run_batch
    problems, refs = _problems()
    n_sm = torch.cuda.get_device_properties(0).multi_processor_count
    alone = run_batch(problems, Plan(parts=1, cap=n_sm, exclusive=[0, 1, 2, 3], groups=[[]]), keep_gradients=True)
    groups, _ = lpt([float(p.shape[0]) for p in problems], 2)
    shared = run_batch(problems, Plan(parts=2, cap=n_sm // 2, exclusive=[], groups=groups), keep_gradients=True)
    for i, (loss_ref, grad_ref) in enumerate(refs):
        g_alone, g_shared = alone["gradients"][i], shared["gradients"][i]
        assert rel(g_shared, g_alone) < 1e-5, i
        assert abs(shared["losses"][i] - loss_ref) / loss_ref < 3e-5, i
        assert rel(g_shared, grad_ref) < 1e-4, i
    # the autotuner's own plan runs and gives the same gradients
    pl = Autotuner(parts=(2, 4), repeats=1).tune(problems, n_sm=n_sm)
    assert sorted(pl.exclusive + [i for g in pl.groups for i in g]) == [0, 1, 2, 3]
    tuned = run_batch(problems, pl, keep_gradients=True)
    for i, (_, grad_ref) in enumerate(refs):
        assert rel(tuned["gradients"][i], grad_ref) < 1e-4, i
    assert tuned["makespan_s"] > 0 and shared["makespan_s"] > 0
