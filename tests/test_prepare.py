"""RF preparation (wust_prepare.m): the oracle pinned to the reference's own
fixture and known answers (Runtime/tests/test_ingest_frequency.m), host-side
validation on CPU, and the GPU DTFT (``wust_dtft``) against the oracle."""
import numpy as np
import pytest

from conftest import gpu_available

GRID = dict(shape_yx=[7, 9], origin_yx_m=[.01, -.02], spacing_yx_m=[.001, .002], origin_kind="pixel_edge")
X = -.02 + (np.arange(9) + .5) * .002
Y_ = .01 + (np.arange(7) + .5) * .001
TX = np.array([[X[2], Y_[2]], [X[5], Y_[4]]])
RX = np.array([TX[0], [X[6], Y_[1]], [X[3], Y_[5]], [X[7], Y_[3]]])


def fixture_rf():
    """test_ingest_frequency.m:92-97: 512 samples from t = 0.7 us, sinusoid
    traces [time, rx, tx], three frequencies."""
    t = np.arange(512) * 1e-7 + 7e-7
    p = np.sin(np.arange(1, 4097) * .17).reshape(512, 4, 2, order="F")
    rf = dict(time_s=t, pressure=p, tx_xy_m=TX, rx_xy_m=RX)
    cfg = dict(grid=GRID, frequencies_hz=[1e5, 2e5, 3e5], c_geom_mps=1500.0, phase_correction="none",
               mask=np.ones((2, 4), bool), data_units="instrument_units", measurement_provenance="fixture")
    return rf, cfg


def test_oracle_geometry_and_dtft_match_reference_known_answers():
    from oracle import prepare_fp64 as o
    _, _, (ti, _), (ri, _) = o.geometry((7, 9), (.01, -.02), (.001, .002), TX, RX)
    assert list(ti) == [17, 40] and list(ri) == [17, 44, 27, 53]          # test_ingest_frequency.m:29
    rf, cfg = fixture_rf()
    Y = o.dtft(rf["time_s"], cfg["frequencies_hz"], rf["pressure"], np.ones((2, 4), bool))
    t = rf["time_s"]
    direct = np.stack([(np.exp(-2j * np.pi * np.asarray(cfg["frequencies_hz"])[:, None] * t[None]) @
                        rf["pressure"][:, :, i] * np.mean(np.diff(t))).astype(np.complex64).T for i in range(2)])
    assert np.linalg.norm(Y - direct) / np.linalg.norm(Y) < 1e-6        # test_ingest_frequency.m:113


@pytest.mark.parametrize("change, message", [
    (lambda rf, cfg: rf.update(time_s=np.r_[rf["time_s"][:-1], rf["time_s"][-1] * 1.01]), "Nonuniform time"),
    (lambda rf, cfg: cfg.update(frequencies_hz=[1e5, 6e6]), "Frequency outside saved Nyquist"),
    (lambda rf, cfg: cfg.update(mask=np.ones((4, 2))), "RF mask must be [tx,rx] or [tx,rx,frequency]"),
    (lambda rf, cfg: cfg.update(mask=np.full((2, 4), 2)), "Mask must contain 0/1"),
    (lambda rf, cfg: rf.update(pressure=rf["pressure"] + 0j), "RF must be real [time,rx,tx] pressure"),
    (lambda rf, cfg: rf.update(tx_xy_m=np.array([[X[2], Y_[2]], [X[2] + 1e-6, Y_[2]]])),
     "Distinct elements in one array collapse onto a grid sample"),
    (lambda rf, cfg: rf.update(tx_xy_m=np.array([[X[0] - .01, Y_[2]], [X[5], Y_[4]]])),
     "Array outside grid sampling coordinates"),
    (lambda rf, cfg: cfg.update(phase_correction="linear"), "Unsupported phase policy"),
    (lambda rf, cfg: cfg.pop("data_units"), "Missing or unsupported RF preparation fields"),
    (lambda rf, cfg: cfg.update(mask=np.zeros((2, 4))), "Empty observations"),
])
def test_prepare_rejects_invalid_input_on_the_host(change, message):
    """Every rejection of wust_prepare.m / wust_geometry.m happens before any
    device work, with WUST:InvalidInput."""
    from waveforminversionust_b200._lib import WustError
    from waveforminversionust_b200.prepare import wust_prepare
    rf, cfg = fixture_rf()
    change(rf, cfg)
    with pytest.raises(WustError) as e:
        wust_prepare(rf, cfg)
    assert e.value.identifier == "WUST:InvalidInput" and message in str(e.value)


@pytest.mark.gpu
@pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")
def test_prepare_fixture_matches_oracle_masks_and_phase():
    from oracle import prepare_fp64 as o
    from waveforminversionust_b200._lib import WustError
    from waveforminversionust_b200.prepare import wust_prepare
    rf, cfg = fixture_rf()
    a = wust_prepare(rf, cfg)
    ref = o.prepare(rf["time_s"], cfg["frequencies_hz"], rf["pressure"], cfg["mask"], (7, 9), (.01, -.02),
                    (.001, .002), TX, RX)
    assert list(a["tx_index"]) == [17, 40] and list(a["rx_index"]) == [17, 44, 27, 53]
    assert a["Y"].dtype == np.complex64 and a["Y"].shape == (2, 4, 3)
    assert np.linalg.norm(a["Y"] - ref["Y"]) / np.linalg.norm(ref["Y"]) < 1e-6
    assert np.array_equal(a["mask"], ref["mask"]) and a["preparation"]["valid_mask_elements"] == 24
    assert a["preparation"]["sampling_interval_s"] == rf["time_s"][1] - rf["time_s"][0]
    # homogeneous time-of-flight phase for off-grid transmitters; norms from the corrected Y
    shifted = dict(rf, tx_xy_m=TX + 1e-4)
    ph = wust_prepare(shifted, dict(cfg, phase_correction="homogeneous-tof"))
    ref = o.prepare(rf["time_s"], cfg["frequencies_hz"], rf["pressure"], cfg["mask"], (7, 9), (.01, -.02),
                    (.001, .002), TX + 1e-4, RX, phase="homogeneous-tof", c_geom=1500.0)
    assert np.linalg.norm(ph["Y"] - ref["Y"]) / np.linalg.norm(ref["Y"]) < 1e-6
    assert np.array_equal(ph["frequency_data_norm"], np.sum(np.abs(ph["Y"].astype(np.complex128)) ** 2, axis=(0, 1)))
    # a masked channel may hold NaN; an active one may not (test_ingest_frequency.m:124-135)
    bad = dict(rf, pressure=rf["pressure"].copy())
    bad["pressure"][:, 0, 0] = np.nan
    m = np.ones((2, 4), bool)
    m[0, 0] = False
    masked = wust_prepare(bad, dict(cfg, mask=m))
    assert np.all(masked["Y"][0, 0, :] == 0) and not masked["mask"][0, 0, :].any()
    with pytest.raises(WustError) as e:
        wust_prepare(bad, cfg)
    assert "Nonfinite RF on an active channel" in str(e.value)


@pytest.mark.gpu
@pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_dtft_ragged_sizes_match_oracle(dtype):
    """700 samples (not a multiple of the 32-sample slab), 9 x 13 traces (not
    a multiple of the 64-trace tile), 37 unsorted frequencies (two frequency
    passes), a [tx, rx, frequency] mask, float64 and float32 RF."""
    from oracle import prepare_fp64 as o
    from waveforminversionust_b200.prepare import dtft_device
    rng = np.random.default_rng(3)
    t = np.arange(700) * 5e-8 - 2e-6
    f = rng.permutation(np.linspace(2e5, 4e6, 37))
    p = rng.standard_normal((700, 13, 9)).astype(dtype)
    active = rng.random((9, 13)) > 0.2
    p[:, ~active.T] = np.nan
    Y = dtft_device(t, f, p, active).cpu().numpy()
    ref = o.dtft(t, f, p.astype(np.float64), active)
    scale = np.abs(ref).max()
    assert np.abs(Y - ref).max() <= 1e-6 * scale
    assert np.all(Y[~active] == 0)
