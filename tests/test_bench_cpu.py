"""Host logic of bench.py's multi-GPU (replica) path on CPU: two gloo ranks."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t = bench.max_over_ranks(10.0 + 5.0 * rank, world, device="cpu")
        out.put((rank, t, bench.aggregate_rate(world, 3, t)))
    finally:
        dist.destroy_process_group()


def test_replica_timing_takes_the_slowest_rank_and_sums_the_work():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, rate in res:
        assert t == 15.0                              # max over ranks, not the local time
        assert abs(rate - 2 * 3 / 15e-3) < 1e-9       # both ranks' gradients over the slowest rank's time


def test_reference_arm_prints_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2")
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--workload", "config1", "--steps", "1",
                        "--warmup", "3"], cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == ""


def test_reference_arm_line_fields():
    """The reference arm (FP64 sparse-LU port on the host cores) prints one
    JSON line with the bench contract's fields."""
    import json
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--workload", "config1", "--steps", "1",
                        "--warmup", "3"], cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["metric"] == "gradients_per_second" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["value"] == line["value"]
    # measured in full on the host cores, and the host is described
    assert line["cpu_baseline"]["cores"] >= 1 and "nothing extrapolated" in line["cpu_baseline"]["sample"]
    assert line["host"]["cpu_count"] >= line["host"]["affinity_cores"] >= 1
    assert abs(line["ms_per_step"] * line["steps"] - 1e3 * line["wall_seconds"]) < 1e-6 * line["ms_per_step"]


def test_batch_problem_mix_follows_the_configuration():
    """The 24 independent inversions of the batch report: interiors from
    {128, 192, 256, 384, 512}, PML 16-20 cells, dx 0.25-0.4 mm, one frequency
    in 0.3-1.2 MHz, transmitters drawn from the ring's receivers, no two ring
    elements on one grid sample, the ring inside the grid."""
    import numpy as np
    import bench
    probs = bench.batch_problems()
    assert len(probs) == 24
    for p in probs:
        ny, nx = p.shape
        assert ny == nx and ny - 2 * p.pml_cells in (128, 192, 256, 384, 512)
        assert 16 <= p.pml_cells <= 20 and 0.25e-3 <= p.dx <= 0.4e-3
        assert p.frequencies_hz.size == 1 and 0.3e6 <= p.frequencies_hz[0] <= 1.2e6
        assert p.tx_index.size in (16, 32, 64, 128, 256) and p.rx_index.size in (32, 64, 128, 256)
        assert p.tx_index.size <= p.rx_index.size
        assert np.unique(p.rx_index).size == p.rx_index.size
        assert np.isin(p.tx_index, p.rx_index).all()
        assert p.rx_index.min() >= 1 and p.rx_index.max() <= ny * nx
        assert p.update_mask.any()
    # the same seed gives the same mix
    again = bench.batch_problems()
    assert all(np.array_equal(a.c_true, b.c_true) and np.array_equal(a.tx_index, b.tx_index)
               for a, b in zip(probs, again))


def test_reconstruction_accepts_correction_precision():
    """correction_precision passes the reconstruction's configuration
    admission (wust_reconstruct.m:124-211 semantics for unknown keys)."""
    import numpy as np
    from waveforminversionust_b200 import synthetic
    from waveforminversionust_b200._lib import WustError
    from waveforminversionust_b200.objective import Observations
    from waveforminversionust_b200.reconstruct import _prepare
    p = synthetic.small(seed=0)
    n_tx, n_rx = p.tx_index.size, p.rx_index.size
    obs = Observations(p.x_m, p.y_m, p.tx_index, p.rx_index, p.frequencies_hz, np.ones((n_tx, n_rx, 1), complex),
                       np.ones((n_tx, n_rx, 1), bool))
    cfg = dict(backend="gpu", bounds_mps=(1300.0, 1800.0), max_update_mps=12.0, step_damping=1.0,
               source_batch_size=4, pml_strength=10.0, pml_m=p.pml_m, stencil_bounds=(1400.0, 1700.0),
               wavenumber="continuum", filter_cutoff=0.0, filter_order=4, update_mask=p.update_mask.astype(float),
               precision="tf32-refined", correction_precision="same")
    assert _prepare(obs, p.c_init, cfg)["correction_precision"] == "same"
    with pytest.raises(WustError):
        _prepare(obs, p.c_init, dict(cfg, correction_precisions="same"))
