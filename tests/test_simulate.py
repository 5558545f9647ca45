"""RF simulation (wust_simulate.m): the FP64 oracle's physics on CPU, host
validation, and the GPU batch against the oracle on the configuration of
the reference's own pipeline test (Runtime/tests/test_native_pipeline.m:
27 x 23 grid, three transmitters, four receivers, 400 samples of a 0.35 MHz
Gaussian-windowed tone, 10-cell PML, c_ref 1550 m/s, decimation by 2, then
the DTFT of wust_prepare at 0.2/0.35/0.45 MHz)."""
import numpy as np
import pytest

from conftest import gpu_available

X = np.arange(-13, 14) * .5e-3
Y = np.arange(-11, 12) * .5e-3


def pipeline_model():
    XX, YY = np.meshgrid(X, Y)
    c = 1500 + 20 * np.exp(-((XX - .001) ** 2 + (YY + .0015) ** 2) / 2e-6)
    ny = Y.size
    sub = lambda r, q: (np.asarray(r) - 1) + ny * (np.asarray(q) - 1) + 1      # MATLAB sub2ind
    dt = 60e-9
    t = np.arange(400) * dt
    return dict(c_mps=c, x_m=X, y_m=Y, tx_index=sub([16, 7, 12], [8, 19, 21]), rx_index=sub([7, 17, 6, 13], [17, 11, 9, 20]),
                dt_s=dt, source_pressure=np.sin(2 * np.pi * .35e6 * t) * np.exp(-((t - 3e-6) / 1e-6) ** 2))


CFG = dict(backend="native-batch", pml_size=10, density_kg_m3=1000, sound_speed_ref_mps=1550, downsample_factor=2,
           time_offset_s=-3e-6)


def test_oracle_physics():
    """Homogeneous medium: the wave front reaches each receiver after
    distance / c (envelope peak of the 3 us-delayed pulse), amplitude falls
    like 1/sqrt(r) in 2-D; the decimation filter has unit DC gain and keeps a
    slow signal."""
    from oracle import kwave_fp64 as k
    c = np.full((23, 27), 1500.0)
    ny = 23
    tx = [7 + ny * 13 + 1]                              # row 8, column 14 (1-based)
    rx = [7 + ny * 23 + 1, 7 + ny * 19 + 1]             # 10 and 6 columns away
    m = pipeline_model()
    out = k.simulate(c, .5e-3, .5e-3, m["dt_s"], m["source_pressure"], tx, rx, 10, 1550, 1000)
    t = np.arange(400) * m["dt_s"]
    peaks = []
    for r, dist in enumerate((5e-3, 3e-3)):
        spec = np.fft.fft(out[r, 0])
        spec[201:] = 0
        spec[1:200] *= 2
        env = np.abs(np.fft.ifft(spec))
        assert abs(t[np.argmax(env)] - (3e-6 + dist / 1500)) < 0.25e-6, r
        peaks.append(env.max())
    assert 0.8 < peaks[0] / peaks[1] * np.sqrt(5 / 3) < 1.25
    h = k.decimation_filter(2)
    assert abs(h.sum() - 1) < 1e-12 and h.size == 97
    slow = np.sin(2 * np.pi * np.arange(400) / 100.0)
    d = k.decimate(slow[None], 2)[0]
    assert np.abs(d[30:170] - slow[60:340:2]).max() < 1e-3


@pytest.mark.parametrize("change, message", [
    (lambda m, c: m.update(dt_s=3e-7), "CFL"),
    (lambda m, c: c.update(sound_speed_ref_mps=1500), "reference speed"),
    (lambda m, c: m.update(tx_index=np.array([5, 5, 9])), "duplicate"),
    (lambda m, c: c.update(downsample_factor=1.5), "decimation"),
    (lambda m, c: c.update(pml_size=0), "PML"),
    (lambda m, c: c.pop("work_dir"), "work_dir"),
    (lambda m, c: m.update(source_pressure=np.array([1.0, np.nan])), "source"),
])
def test_simulate_rejects_what_the_reference_rejects(tmp_path, change, message):
    from waveforminversionust_b200 import WustError
    from waveforminversionust_b200.simulate import wust_simulate
    m, c = pipeline_model(), dict(CFG, work_dir=str(tmp_path))
    change(m, c)
    with pytest.raises(WustError, match=message):
        wust_simulate(m, c)


@pytest.mark.gpu
@pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")
def test_simulation_matches_the_oracle_on_the_reference_pipeline_case(tmp_path):
    from oracle import kwave_fp64 as k
    from waveforminversionust_b200.prepare import wust_prepare
    from waveforminversionust_b200.simulate import wust_simulate
    m = pipeline_model()
    batch = wust_simulate(m, dict(CFG, work_dir=str(tmp_path)))
    serial = wust_simulate(m, dict(CFG, backend="matlab-serial", work_dir=str(tmp_path)))
    full = wust_simulate(m, dict(CFG, downsample_factor=1, work_dir=str(tmp_path)))
    ref = k.simulate(m["c_mps"], .5e-3, .5e-3, m["dt_s"], m["source_pressure"], m["tx_index"], m["rx_index"], 10, 1550,
                     1000)                                                    # [rx, tx, time]
    want_full = np.transpose(ref, (2, 0, 1))
    rel = lambda a, b: np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel())
    assert full["pressure"].shape == (400, 4, 3) and batch["pressure"].shape == (200, 4, 3)
    assert rel(full["pressure"], want_full) < 1e-4
    want = np.transpose(k.decimate(ref, 2), (2, 0, 1))
    assert rel(batch["pressure"], want) < 1e-4
    assert rel(batch["pressure"], serial["pressure"]) < 1e-6                  # test_native_pipeline.m: 1e-4
    assert np.abs(batch["time_s"] - (np.arange(200) * 120e-9 - 3e-6)).max() < 1e-15
    assert np.array_equal(batch["tx_xy_m"], serial["tx_xy_m"])
    grid = dict(shape_yx=[23, 27], spacing_yx_m=[.0005, .0005], origin_yx_m=[Y[0] - .00025, X[0] - .00025],
                origin_kind="pixel_edge")
    prep = dict(frequencies_hz=[.2e6, .35e6, .45e6], grid=grid, c_geom_mps=1500, phase_correction="none",
                mask=np.ones((3, 4), bool), data_units="Pa*s", measurement_provenance="self_simulated")
    dn = wust_prepare(batch, prep)
    ds = wust_prepare(serial, prep)
    assert rel(dn["Y"], ds["Y"]) < 1e-4
    assert np.array_equal(dn["tx_index"], m["tx_index"]) and np.array_equal(dn["rx_index"], m["rx_index"])
