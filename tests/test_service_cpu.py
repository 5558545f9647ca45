"""The runtime service on CPU: request and manifest rules of the reference's
transport (Runtime/python/contracts.py, wust_io.py), artifact round trips,
the ingest_frequency operation end to end through the supervised worker
(wust_run.m:7-9 with wust_prepare_observations.m), failures and the
deadline.

Without h5py on this host the array files go through the stand-in module
in tests/h5stub (an .npz archive per "HDF5" file), on the worker's path
too; with h5py present the real files are written."""
import importlib.util
import json
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
STUB = os.path.join(HERE, "h5stub")
HAVE_H5PY = importlib.util.find_spec("h5py") is not None       # decided before the stand-in is imported

GRID = dict(shape_yx=[30, 36], origin_yx_m=[-.015, -.018], spacing_yx_m=[.001, .001], origin_kind="pixel_edge")
XS = -.018 + (np.arange(36) + .5) * .001
YS = -.015 + (np.arange(30) + .5) * .001
TX = np.array([[XS[5], YS[6]], [XS[20], YS[24]], [XS[30], YS[10]]])
RX = np.array([[XS[3], YS[3]], [XS[33], YS[4]], [XS[18], YS[27]], [XS[10], YS[15]], [XS[25], YS[20]]])


@pytest.fixture()
def transport(monkeypatch):
    if not HAVE_H5PY:
        monkeypatch.syspath_prepend(STUB)
        monkeypatch.setenv("PYTHONPATH", STUB + os.pathsep + os.environ.get("PYTHONPATH", ""))
    from waveforminversionust_b200 import transport as T
    return T


def request(op, inp, out, config=None, **extra):
    return dict(schema="wust.request", schema_version=2, operation=op, input_manifest=str(inp),
                output_manifest=str(out), config={} if config is None else config, **extra)


def frequency_input(seed=0):
    """A frequency input in the [frequency, tx, rx] order with Fourier sign
    +1 (real time-domain pressure declared), unsorted frequencies and a
    [tx, rx] mask."""
    rng = np.random.default_rng(seed)
    f = np.array([6e5, 3e5, 4.5e5])
    p = (rng.standard_normal((3, 3, 5)) + 1j * rng.standard_normal((3, 3, 5))).astype(np.complex64)
    mask = np.ones((3, 5), bool)
    mask[1, 2] = False
    meta = dict(grid=GRID, pressure_type="total_pressure", data_units="instrument_units",
                spectrum_normalization="unknown", fourier_sign=1, real_pressure=True,
                measurement_provenance="synthetic")
    arrays = dict(frequencies_hz=f, tx_xy_m=TX, rx_xy_m=RX, pressure=p, mask=mask)
    return meta, arrays, dict(pressure="frequency,tx,rx", mask="tx,rx")


def test_request_rules(transport):
    T = transport
    ok = request("reconstruct", "/a.json", "/b.json", dict(backend="gpu"), initial_manifest="/c.json",
                 frequency_schedule_hz=[3e5], max_updates=2, save_history=False)
    assert T.validate_request(ok) is ok
    bad = [
        dict(ok, schema_version=True),                           # bool is not the integer 2
        dict(ok, schema="wust.rf"),
        {k: v for k, v in ok.items() if k != "initial_manifest"},
        dict(ok, max_updates=-1),
        dict(ok, max_updates=1.0),
        dict(ok, frequency_schedule_hz=[0.0]),
        dict(ok, frequency_schedule_hz=[float("inf")]),
        dict(ok, save_history=1),
        dict(ok, operation="fit"),
        dict(ok, extra=1),
        request("prepare", "/a", "/b", {}, max_updates=1),        # controls only on reconstruct
        request("ingest_frequency", "/a", "/b", {"x": 1}),        # ingest takes an empty config
    ]
    for req in bad:
        with pytest.raises(ValueError):
            T.validate_request(req)


def test_artifact_round_trip_and_manifest_rules(transport, tmp_path):
    T = transport
    meta, arrays, axes = frequency_input()
    path = tmp_path / "input.json"
    doc = T.write_artifact(path, "wust.frequency_input", meta, arrays, axes)
    assert doc["arrays"]["pressure"]["real_dataset"] == "/pressure_real"
    assert doc["arrays"]["mask"]["dtype"] == "bool" and doc["arrays"]["pressure"]["units"] == "instrument_units"
    got_doc, got = T.read_artifact(path, "wust.frequency_input")
    assert got_doc["metadata"]["fourier_sign"] == 1
    for k, v in arrays.items():
        assert got[k].dtype == v.dtype and np.array_equal(got[k], v), k
    with pytest.raises(FileExistsError):
        T.write_artifact(path, "wust.frequency_input", meta, arrays, axes)
    with pytest.raises(ValueError):
        T.read_manifest(path, "wust.measurements")              # another schema expected

    def broken(edit, name):
        d = json.loads(path.read_text())
        edit(d)
        p = tmp_path / name
        p.write_text(json.dumps(d))
        with pytest.raises((ValueError, FileNotFoundError)):
            T.read_manifest(p)

    broken(lambda d: d["arrays"]["pressure"].update(real_dataset="/p_real"), "names.json")
    broken(lambda d: d["arrays"]["pressure"].update(shape=[3, 3]), "rank.json")
    broken(lambda d: d["arrays"]["pressure"].update(shape=[3, 3, 0]), "zero.json")
    broken(lambda d: d["arrays"]["mask"].update(axes="rx,tx"), "axes.json")
    broken(lambda d: d["arrays"]["pressure"].update(units="Pa"), "units.json")
    broken(lambda d: d.update(arrays_file="../input.h5"), "sibling.json")
    broken(lambda d: d["arrays"].pop("mask"), "missing.json")
    broken(lambda d: d.update(extra=1), "extra.json")
    # a descriptor that disagrees with the stored dataset is caught on read
    d = json.loads(path.read_text())
    d["arrays"]["pressure"]["dtype"] = "complex128"
    (tmp_path / "dtype.json").write_text(json.dumps(d))
    with pytest.raises(ValueError, match="differs"):
        T.read_artifact(tmp_path / "dtype.json")


def test_ingest_frequency_through_the_service(transport, tmp_path):
    T = transport
    from waveforminversionust_b200 import service
    from waveforminversionust_b200.prepare import wust_geometry
    meta, arrays, axes = frequency_input(seed=3)
    inp = tmp_path / "input.json"
    T.write_artifact(inp, "wust.frequency_input", meta, arrays, axes)
    req = tmp_path / "request.json"
    out = tmp_path / "out" / "measurements.json"
    out.parent.mkdir()
    req.write_text(json.dumps(request("ingest_frequency", inp, out)))
    result = service.run(req, timeout_s=300)
    assert out.is_file() and result["schema"] == "wust.measurements"
    assert (out.parent / result["arrays_file"]).is_file()
    assert not any(p.name == "result.json" for p in out.parent.rglob("*"))
    doc, got = T.read_artifact(out, "wust.measurements")
    # wust_prepare_observations: [tx, rx, frequency], conjugated (sign +1),
    # ascending frequencies, masked entries zero, geometry snapped
    order = np.argsort(arrays["frequencies_hz"])
    want = np.conj(np.moveaxis(arrays["pressure"], 0, 2))[:, :, order]
    want[~arrays["mask"]] = 0
    assert np.array_equal(got["frequencies_hz"], arrays["frequencies_hz"][order])
    assert got["Y"].dtype == np.complex64 and np.array_equal(got["Y"], want)
    assert got["mask"].shape == (3, 5, 3) and not got["mask"][1, 2].any() and got["mask"].sum() == 14 * 3
    geo = wust_geometry(GRID, TX, RX)
    assert np.array_equal(got["tx_index"], geo["tx_index"]) and np.array_equal(got["rx_index"], geo["rx_index"])
    md = doc["metadata"]
    assert md["fourier_sign"] == -1 and md["preparation"]["conversion"] == "conjugate"
    assert md["preparation"]["canonical_to_input_permutation_1based"] == list(order + 1)
    assert "shape_yx" not in md and "frequency_data_norm" not in md       # derived fields are not written
    assert md["runtime_version"] == service.RUNTIME_VERSION and md["request_timeout_s"] == 300
    # the canonical artifact is accepted as canonical input: same observations
    from waveforminversionust_b200.prepare import wust_prepare_observations
    again = wust_prepare_observations(service._artifact_value(out, "wust.measurements"))
    assert np.array_equal(again["Y"], got["Y"]) and np.array_equal(again["mask"], got["mask"])


def test_service_failures(transport, tmp_path):
    T = transport
    from waveforminversionust_b200 import service
    meta, arrays, axes = frequency_input()
    meta = dict(meta, pressure_type="scattered_pressure")
    inp = tmp_path / "input.json"
    T.write_artifact(inp, "wust.frequency_input", meta, arrays, axes)
    req = tmp_path / "request.json"
    req.write_text(json.dumps(request("ingest_frequency", inp, tmp_path / "out.json")))
    with pytest.raises(service.RuntimeFailure) as err:
        service.run(req, timeout_s=300)
    assert err.value.reason == "runtime_failure" and "total complex pressure" in str(err.value)
    assert not (tmp_path / "out.json").exists()
    runs = [p for p in tmp_path.iterdir() if p.is_dir() and "-run-" in p.name]
    assert runs and (runs[0] / "failure.json").is_file()          # kept for diagnosis
    fail = json.loads((runs[0] / "failure.json").read_text())
    assert fail["schema"] == "wust.execution_failure" and fail["identifier"] == "WUST:InvalidInput"
    # the deadline ends the worker's process group
    req2 = tmp_path / "request2.json"
    req2.write_text(json.dumps(request("ingest_frequency", inp, tmp_path / "out2.json")))
    with pytest.raises(service.RuntimeFailure) as err:
        service.run(req2, timeout_s=0.05)
    assert err.value.reason == "time_budget"
    # transport errors before any work: relative paths, an existing output, no timeout
    with pytest.raises(ValueError, match="absolute"):
        (tmp_path / "r3.json").write_text(json.dumps(request("ingest_frequency", "input.json", tmp_path / "o3.json")))
        service.run(tmp_path / "r3.json", timeout_s=10)
    (tmp_path / "exists.json").write_text("{}")
    (tmp_path / "r4.json").write_text(json.dumps(request("ingest_frequency", inp, tmp_path / "exists.json")))
    with pytest.raises(FileExistsError):
        service.run(tmp_path / "r4.json", timeout_s=10)
    with pytest.raises(ValueError, match="timeout_s"):
        service.run(tmp_path / "r4.json", timeout_s=None)


def test_describe_command_line(transport):
    import subprocess
    out = subprocess.run([sys.executable, "-m", "waveforminversionust_b200.service", "describe"], capture_output=True,
                         text=True, check=True, cwd=os.path.dirname(HERE))
    caps = json.loads(out.stdout)
    assert caps["schema"] == "wust.capabilities" and caps["schema_version"] == 2
    assert set(caps["operations"]) == {"ingest_frequency", "prepare", "reconstruct", "simulate"}
    assert caps["fourier_sign"] == -1
