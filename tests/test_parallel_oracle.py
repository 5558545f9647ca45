"""The host-parallel FP64 gradient (CPU baseline and full-size parity reference)
equals the serial FP64 oracle (to rounding: each worker factors its own operator
with one BLAS thread): splitting the transmitters over worker
processes is wust_oracle's batch invariance (Runtime/tests/test_runtime.m:57-61)."""
import numpy as np


def test_parallel_gradient_matches_serial_oracle():
    from oracle import helmholtz_fp64 as o
    from oracle.parallel_fp64 import ParallelOracle
    from waveforminversionust_b200 import synthetic
    p = synthetic.small(seed=2, n_tx=5)
    ny, nx = p.shape
    f = float(p.frequencies_hz[0])
    n_tx, n_rx = p.tx_index.size, p.rx_index.size
    dummy = o.Observations(p.x_m, p.y_m, p.tx_index, p.rx_index, [f], np.zeros((n_tx, n_rx, 1)),
                           np.ones((n_tx, n_rx, 1), bool))
    cfg = o.OracleConfig(pml_m=p.pml_m)
    u = o.make_solver(p.c_true, dummy, 0, cfg).solve(o.point_sources(p.tx_index, range(n_tx), ny, nx))
    Y = u.reshape(-1, n_tx, order="F")[p.rx_index - 1, :].T
    mask = np.ones((n_tx, n_rx), bool)
    mask[1, :3] = False
    obs = o.Observations(p.x_m, p.y_m, p.tx_index, p.rx_index, [f], Y[:, :, None], mask[:, :, None])
    loss, grad, cache = o.wust_oracle(p.c_init, obs, 0, cfg, retain_state=True)
    with ParallelOracle(workers=2) as pool:
        out = pool.gradient(p.x_m, p.y_m, p.c_init, f, p.pml_m, p.tx_index, p.rx_index, Y, mask, keep_fields=(0, 4))
    assert out["workers"] == 2
    assert abs(out["loss"] - loss) <= 1e-12 * loss
    assert np.linalg.norm(out["gradient"] - grad) <= 1e-10 * np.linalg.norm(grad)
    for k in (0, 4):
        want = cache["fields"][0][:, :, k]
        assert np.linalg.norm(out["fields"][k] - want) <= 1e-8 * np.linalg.norm(want)
