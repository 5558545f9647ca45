import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def ref_fixture():
    """The 31 x 31 coherent fixture of Runtime/tests/test_runtime.m:10-17 and
    Runtime/tests/wust_test_measurements.m:12-35 (3 TX, 4 RX, 0.1/0.12 MHz,
    observations generated by the FP64 solver on the true model)."""
    from oracle import helmholtz_fp64 as o
    x = np.arange(-15, 16) * 1e-3
    xg, yg = o.grid_centres((31, 31), (-.0155, -.0155), (.001, .001))
    txy = np.stack([x[[7, 22, 24]], x[[9, 21, 15]]], 1)
    rxy = np.stack([x[[12, 23, 14, 7]], x[[7, 14, 22, 17]]], 1)
    tx = o.snap(txy, xg, yg)
    rx = o.snap(rxy, xg, yg)
    X, Y = np.meshgrid(xg, yg)
    c_true = 1500 + 30 * np.exp(-(X ** 2 + Y ** 2) / 3e-5)
    freqs = np.array([1e5, 1.2e5])
    cfg = o.OracleConfig(pml_m=.004, pml_strength=10, stencil_bounds=(1400, 1700), source_batch_size=2)
    Yobs = np.zeros((3, 4, 2), complex)
    dummy = o.Observations(xg, yg, tx, rx, freqs, np.zeros((3, 4, 2)), np.ones((3, 4, 2), bool))
    for fi in range(2):
        s = o.make_solver(c_true, dummy, fi, cfg)
        u = s.solve(o.point_sources(tx, range(3), 31, 31))
        Yobs[:, :, fi] = u.reshape(-1, 3, order="F")[rx - 1, :].T
    obs = o.Observations(xg, yg, tx, rx, freqs, Yobs, np.ones((3, 4, 2), bool))
    mask = np.ones((31, 31), bool)
    mask[[*range(5), *range(26, 31)], :] = False
    mask[:, [*range(5), *range(26, 31)]] = False
    direction = np.exp(-((X - .002) ** 2 + (Y + .003) ** 2) / 2e-5) * mask * 1e-6
    return dict(x=xg, y=yg, X=X, Y=Y, tx=tx, rx=rx, c_true=c_true, freqs=freqs, obs=obs, cfg=cfg, mask=mask,
                direction=direction, initial=1500 * np.ones((31, 31)))
