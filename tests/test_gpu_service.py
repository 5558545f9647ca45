"""The runtime service's GPU operations against direct library calls:
``reconstruct`` (wust_run.m:20-32: observations from a measurements
artifact, initial model and update mask from an initial-model artifact, the
request's schedule controls) and ``prepare`` (wust_run.m:11-19, the DTFT on
the GPU), each run through the supervised worker process and compared with
the same computation made in this process."""
import json

import numpy as np
import pytest

from conftest import gpu_available
from test_service_cpu import request, transport  # noqa: F401  (fixture)

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]


def _grid_of(p):
    dx, dy = p.x_m[1] - p.x_m[0], p.y_m[1] - p.y_m[0]
    return dict(shape_yx=[int(p.y_m.size), int(p.x_m.size)], origin_yx_m=[float(p.y_m[0] - dy / 2),
                float(p.x_m[0] - dx / 2)], spacing_yx_m=[float(dy), float(dx)], origin_kind="pixel_edge")


def _xy_of(p, index):
    iy, ix = (index - 1) % p.y_m.size, (index - 1) // p.y_m.size
    return np.stack([p.x_m[ix], p.y_m[iy]], axis=1)


def test_reconstruct_through_the_service_matches_the_direct_loop(transport, tmp_path):  # noqa: F811
    T = transport
    from oracle import helmholtz_fp64 as o
    from waveforminversionust_b200 import service, synthetic
    from waveforminversionust_b200.objective import POOL, Observations
    from waveforminversionust_b200.reconstruct import wust_reconstruct
    p = synthetic._problem("recon80", 64, 8, 0.5e-3, 32, 14e-3, 8, [0.25e6, 0.35e6],
                           lambda X, Y: 1500 + 25 * np.exp(-((X - 2e-3) ** 2 + Y ** 2) / (2 * (4e-3) ** 2)), 12e-3)
    ny, nx = p.shape
    n_tx, n_rx, nf = p.tx_index.size, p.rx_index.size, p.frequencies_hz.size
    ocfg = o.OracleConfig(pml_m=p.pml_m, pml_strength=10, stencil_bounds=(1400, 1700), source_batch_size=4)
    dummy = o.Observations(p.x_m, p.y_m, p.tx_index, p.rx_index, p.frequencies_hz, np.zeros((n_tx, n_rx, nf)),
                           np.ones((n_tx, n_rx, nf), bool))
    Y = np.zeros((n_tx, n_rx, nf), np.complex64)
    for fi in range(nf):
        u = o.make_solver(p.c_true, dummy, fi, ocfg).solve(o.point_sources(p.tx_index, range(n_tx), ny, nx))
        Y[:, :, fi] = u.reshape(-1, n_tx, order="F")[p.rx_index - 1, :].T
    mask = np.ones((n_tx, n_rx, nf), bool)
    meas = tmp_path / "measurements.json"
    T.write_artifact(meas, "wust.measurements",
                     dict(grid=_grid_of(p), fourier_sign=-1, data_units="instrument_units",
                          spectrum_normalization="unknown", pressure_type="total_pressure"),
                     dict(frequencies_hz=p.frequencies_hz, tx_xy_m=_xy_of(p, p.tx_index), rx_xy_m=_xy_of(p, p.rx_index),
                          Y=Y, mask=mask, tx_index=p.tx_index.astype(np.int64), rx_index=p.rx_index.astype(np.int64)))
    init = tmp_path / "initial.json"
    T.write_artifact(init, "wust.initial_model", {}, dict(initial_mps=p.c_init, update_mask=p.update_mask))
    config = dict(backend="gpu", bounds_mps=[1400.0, 1700.0], max_update_mps=12.0, step_damping=1.0,
                  source_batch_size=4, pml_strength=10.0, pml_m=p.pml_m, stencil_bounds=[1400.0, 1700.0],
                  wavenumber="continuum", filter_cutoff=0.0, filter_order=4, precision="tf32-refined")
    schedule = [float(p.frequencies_hz[0]), float(p.frequencies_hz[1]), float(p.frequencies_hz[1])]
    out = tmp_path / "recon.json"
    req = tmp_path / "request.json"
    req.write_text(json.dumps(request("reconstruct", meas, out, config, initial_manifest=str(init),
                                      frequency_schedule_hz=schedule, max_updates=3, save_history=True)))
    result = service.run(req, timeout_s=600)
    doc, arrays = T.read_artifact(out, "wust.reconstruction")
    md = doc["metadata"]
    assert md["completed_updates"] == 3 and md["executed_schedule"] == [1, 2, 2]
    assert md["executed_frequencies_hz"] == schedule and len(md["records"]) == 3
    assert md["environment"]["precision_profile"] == "tf32-refined" and "B200" in md["environment"]["gpu_device"]
    assert arrays["history_mps"].shape == (ny, nx, 4) and arrays["history_mps"].dtype == np.float32
    assert result["arrays_file"].endswith(".h5")

    cfg = dict(config, update_mask=p.update_mask, frequency_schedule_hz=schedule, max_updates=3)
    obs = Observations(p.x_m, p.y_m, p.tx_index, p.rx_index, p.frequencies_hz, Y, mask)
    direct = wust_reconstruct(obs, p.c_init, cfg)
    POOL.clear()
    moved = np.abs(direct["c_mps"] - p.c_init).max()
    assert moved > 1.0
    assert np.abs(arrays["c_mps"] - direct["c_mps"]).max() <= 1e-6 * moved
    for r_s, r_d in zip(md["records"], direct["records"]):
        assert abs(r_s["loss_before_update"] - r_d["loss_before_update"]) <= 1e-9 * abs(r_d["loss_before_update"])


def test_prepare_through_the_service_matches_wust_prepare(transport, tmp_path):  # noqa: F811
    T = transport
    from test_prepare import GRID, RX, TX
    from waveforminversionust_b200 import service
    from waveforminversionust_b200.prepare import wust_prepare
    rng = np.random.default_rng(5)
    t = np.arange(900) * 5e-8 + 1e-6
    rf = dict(time_s=t, pressure=rng.standard_normal((900, 4, 2)), tx_xy_m=TX, rx_xy_m=RX)
    rf_art = tmp_path / "rf.json"
    T.write_artifact(rf_art, "wust.rf", dict(data_units="Pa", measurement_provenance="synthetic"), rf)
    config = dict(grid=GRID, frequencies_hz=[2e5, 1e5, 3e5], c_geom_mps=1500.0, phase_correction="homogeneous-tof",
                  mask=[[True, True, False, True], [True, True, True, True]])
    out = tmp_path / "meas.json"
    req = tmp_path / "request.json"
    req.write_text(json.dumps(request("prepare", rf_art, out, config)))
    service.run(req, timeout_s=600)
    doc, arrays = T.read_artifact(out, "wust.measurements")
    want = wust_prepare(rf, dict(config, mask=np.array(config["mask"]), data_units="Pa*s",
                                 measurement_provenance="synthetic"))
    assert doc["metadata"]["data_units"] == "Pa*s" and doc["metadata"]["preparation"]["phase_correction"] == \
        "homogeneous-tof"
    assert np.array_equal(arrays["frequencies_hz"], want["frequencies_hz"])
    assert np.array_equal(arrays["mask"], want["mask"])
    scale = np.abs(want["Y"]).max()
    assert np.abs(arrays["Y"] - want["Y"]).max() <= 1e-6 * scale


def test_simulate_through_the_service_matches_wust_simulate(transport, tmp_path):  # noqa: F811
    """wust_run.m:33-39: the simulation input's positions snapped to its grid,
    then wust_simulate; the RF artifact against the direct call."""
    T = transport
    from test_simulate import CFG, X, Y, pipeline_model
    from waveforminversionust_b200 import service
    from waveforminversionust_b200.simulate import wust_simulate
    m = pipeline_model()
    ny = Y.size
    iy, ix = (m["tx_index"] - 1) % ny, (m["tx_index"] - 1) // ny
    ry, rx = (m["rx_index"] - 1) % ny, (m["rx_index"] - 1) // ny
    grid = dict(shape_yx=[23, 27], spacing_yx_m=[.0005, .0005], origin_yx_m=[Y[0] - .00025, X[0] - .00025],
                origin_kind="pixel_edge")
    inp = tmp_path / "model.json"
    T.write_artifact(inp, "wust.simulation_input", dict(grid=grid, dt_s=m["dt_s"]),
                     dict(c_mps=m["c_mps"], tx_xy_m=np.stack([X[ix], Y[iy]], 1), rx_xy_m=np.stack([X[rx], Y[ry]], 1),
                          source_pressure=m["source_pressure"]))
    cfg = dict(CFG, work_dir=str(tmp_path / "work"))
    out = tmp_path / "rf.json"
    req = tmp_path / "request.json"
    req.write_text(json.dumps(request("simulate", inp, out, cfg)))
    service.run(req, timeout_s=600)
    doc, arrays = T.read_artifact(out, "wust.rf")
    want = wust_simulate(m, cfg)
    assert doc["metadata"]["data_units"] == "Pa" and doc["metadata"]["measurement_provenance"] == "self_simulated"
    assert arrays["pressure"].shape == (200, 4, 3) and arrays["pressure"].dtype == np.float32
    assert np.abs(arrays["pressure"] - want["pressure"]).max() <= 1e-6 * np.abs(want["pressure"]).max()
    assert np.array_equal(arrays["time_s"], want["time_s"])
    # the service takes the grid positions from the artifact's grid, the direct call from the test's axes
    assert np.allclose(arrays["tx_xy_m"], want["tx_xy_m"], rtol=0, atol=1e-12)
    assert np.allclose(arrays["rx_xy_m"], want["rx_xy_m"], rtol=0, atol=1e-12)
