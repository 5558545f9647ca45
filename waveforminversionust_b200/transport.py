"""WUST v2 transport: requests, JSON manifests and their HDF5 array files.

This is the file contract of the reference's Python runtime
(Runtime/python/contracts.py:1-186 for the schemas and the request rules,
Runtime/python/wust_io.py:1-169 for manifests and array files, and the
MATLAB side that fills them, Runtime/matlab/wust_read_artifact.m:1-67 and
wust_write_artifact.m:1-89), restated so that a caller of the reference's
runtime can point the same request files at this library.

An artifact is a JSON manifest (schema name, version 2, free-form metadata,
the name of a sibling HDF5 file and one descriptor per array) next to that
HDF5 file, which holds each array once in its declared axis order (complex
arrays as separate ``<name>_real`` / ``<name>_imag`` datasets, booleans as
uint8 0/1).  The manifest is published last and atomically, so it is the
success index of a run.  HDF5 goes through ``h5py``, as in the reference
(it is imported only when arrays are read or written, and a missing h5py is
reported as a runtime failure).
"""
from __future__ import annotations

import json
import math
import os
import tempfile
from dataclasses import dataclass
from pathlib import Path

import numpy as np

PROTOCOL_VERSION = 2


class TransportError(ValueError):
    """A request or artifact that breaks the contract; ``reason`` is the
    failure category of a ``wust.execution_failure`` document."""

    def __init__(self, message: str, reason: str = "incompatible_request"):
        super().__init__(message)
        self.reason = reason


@dataclass(frozen=True)
class ArrayField:
    axes: tuple          # accepted axis strings, e.g. ("tx,rx,frequency",)
    units: str           # "data_units": the artifact's metadata.data_units
    dtypes: tuple
    optional: bool = False


_REAL = ("float32", "float64")
_COMPLEX = ("complex64", "complex128")
_MASK = ("bool", "uint8")
_GEOMETRY = {
    "frequencies_hz": ArrayField(("frequency",), "Hz", _REAL),
    "tx_xy_m": ArrayField(("tx,xy",), "m", _REAL),
    "rx_xy_m": ArrayField(("rx,xy",), "m", _REAL),
}

# The array fields of every artifact schema (contracts.py:31-64).
ARRAY_FIELDS = {
    "wust.frequency_input": {
        **_GEOMETRY,
        "pressure": ArrayField(("frequency,tx,rx", "tx,rx,frequency"), "data_units", _COMPLEX),
        "mask": ArrayField(("frequency,tx,rx", "tx,rx,frequency", "tx,rx"), "1", _MASK),
    },
    "wust.measurements": {
        **_GEOMETRY,
        "Y": ArrayField(("tx,rx,frequency",), "data_units", _COMPLEX),
        "mask": ArrayField(("tx,rx,frequency",), "1", _MASK),
        "tx_index": ArrayField(("tx",), "1", ("int64", "float64")),
        "rx_index": ArrayField(("rx",), "1", ("int64", "float64")),
    },
    "wust.initial_model": {
        "initial_mps": ArrayField(("y,x",), "m/s", _REAL),
        "update_mask": ArrayField(("y,x",), "1", _MASK),
    },
    "wust.reconstruction": {
        "c_mps": ArrayField(("y,x",), "m/s", ("float64",)),
        "history_mps": ArrayField(("y,x,model_step",), "m/s", ("float32",), optional=True),
    },
    "wust.rf": {
        "pressure": ArrayField(("time,rx,tx",), "data_units", _REAL),
        "time_s": ArrayField(("time",), "s", _REAL),
        "tx_xy_m": _GEOMETRY["tx_xy_m"],
        "rx_xy_m": _GEOMETRY["rx_xy_m"],
    },
    "wust.simulation_input": {
        "c_mps": ArrayField(("y,x",), "m/s", _REAL),
        "tx_xy_m": _GEOMETRY["tx_xy_m"],
        "rx_xy_m": _GEOMETRY["rx_xy_m"],
        "source_pressure": ArrayField(("time",), "Pa", _REAL),
    },
}
SCHEMAS = {name: PROTOCOL_VERSION for name in
           (*ARRAY_FIELDS, "wust.request", "wust.capabilities", "wust.execution_failure")}

# Input schemas of each operation, and the schema of its result.
OPERATION_INPUTS = {
    "ingest_frequency": ("wust.frequency_input",),
    "prepare": ("wust.rf",),
    "reconstruct": ("wust.frequency_input", "wust.measurements"),
    "simulate": ("wust.simulation_input",),
}
OPERATION_OUTPUT = {"ingest_frequency": "wust.measurements", "prepare": "wust.measurements",
                    "reconstruct": "wust.reconstruction", "simulate": "wust.rf"}

_BASE_REQUEST = ("schema", "schema_version", "operation", "input_manifest", "output_manifest", "config")
_RECONSTRUCTION_REQUEST = ("initial_manifest", "frequency_schedule_hz", "max_updates", "save_history")
_MANIFEST_KEYS = ("schema", "schema_version", "metadata", "arrays_file", "arrays")

# Prepared quantities that a reader rebuilds from the canonical arrays; they
# are not written into a manifest's metadata (wust_write_artifact.m:8-14).
DERIVED_FIELDS = ("x_m", "y_m", "tx_snapped_xy_m", "rx_snapped_xy_m", "pressure_axes", "mask_axes", "shape_yx",
                  "n_tx", "n_rx", "valid_receiver_counts", "frequency_data_norm")


def require_keys(value, required, optional=()) -> None:
    """``value`` is an object holding every required key and nothing else
    than the optional ones."""
    if not isinstance(value, dict):
        raise TransportError("Expected an object")
    have = set(value)
    missing, unknown = set(required) - have, have - set(required) - set(optional)
    if missing or unknown:
        raise TransportError(f"Missing fields {sorted(missing)}; unsupported fields {sorted(unknown)}")


def check_envelope(doc, expected=None) -> None:
    """Schema name known (and among ``expected``, a name or a tuple of names)
    and schema_version the integer 2 (bool is not an integer here)."""
    if not isinstance(doc, dict):
        raise TransportError("Schema envelope must be an object")
    name = doc.get("schema")
    accepted = (expected,) if isinstance(expected, str) else expected
    if not isinstance(name, str) or name not in SCHEMAS or (accepted is not None and name not in accepted):
        raise TransportError(f"Unsupported schema {name!r}; expected {expected}")
    version = doc.get("schema_version")
    if type(version) is not int or version != PROTOCOL_VERSION:
        raise TransportError("schema_version must be integer 2")


def check_number(value, label: str, minimum: float = 0.0, inclusive: bool = False) -> None:
    if type(value) not in (int, float) or not math.isfinite(value):
        raise TransportError(f"{label} must be a finite real number")
    if value < minimum or (value == minimum and not inclusive):
        raise TransportError(f"{label} outside its legal range")


def validate_request(req) -> dict:
    """The request rules of contracts.py:134-162: exact keys, a known
    operation with an object config, the reconstruction controls only on
    reconstruct (where the initial model is required), an empty config for
    ingest_frequency."""
    check_envelope(req, "wust.request")
    require_keys(req, _BASE_REQUEST, _RECONSTRUCTION_REQUEST)
    if req["operation"] not in OPERATION_INPUTS or not isinstance(req["config"], dict):
        raise TransportError("Unsupported operation/config")
    if req["operation"] == "reconstruct":
        if "initial_manifest" not in req:
            raise TransportError("Reconstruction requires an explicit initial model")
        schedule = req.get("frequency_schedule_hz")
        if schedule is not None:
            if not isinstance(schedule, list):
                raise TransportError("frequency_schedule_hz must be a list or null")
            for f in schedule:
                check_number(f, "frequency_schedule_hz")
        cap = req.get("max_updates")
        if cap is not None and (type(cap) is not int or cap < 0):
            raise TransportError("max_updates must be a nonnegative integer or null")
        if type(req.get("save_history", False)) is not bool:
            raise TransportError("save_history must be boolean")
    elif set(_RECONSTRUCTION_REQUEST) & set(req):
        raise TransportError("Initial model and update controls belong only to reconstruction")
    if req["operation"] == "ingest_frequency":
        require_keys(req["config"], ())
    return req


def read_json(path):
    with Path(path).open(encoding="utf-8") as stream:
        return json.load(stream)


def to_json(value):
    """Metadata in JSON terms: arrays and NumPy scalars to lists and Python
    numbers, non-finite numbers to null (MATLAB's jsonencode writes NaN as
    null), tuples to lists."""
    if isinstance(value, dict):
        return {str(k): to_json(v) for k, v in value.items()}
    if isinstance(value, (list, tuple)):
        return [to_json(v) for v in value]
    if isinstance(value, np.ndarray):
        return to_json(value.tolist())
    if isinstance(value, (np.bool_, bool)):
        return bool(value)
    if isinstance(value, (np.integer,)):
        return int(value)
    if isinstance(value, (float, np.floating)):
        v = float(value)
        return v if math.isfinite(v) else None
    if isinstance(value, (complex, np.complexfloating)):
        raise TransportError("complex values belong in arrays, not metadata")
    return value


def atomic_json(path, value) -> None:
    """Write ``value`` to a new file ``path`` all at once (temporary file in
    the same folder, fsync, rename); an existing file is never replaced."""
    path = Path(path)
    if path.exists():
        raise FileExistsError(path)
    fd, tmp = tempfile.mkstemp(dir=path.parent, prefix=f".{path.name}.", suffix=".tmp")
    try:
        with os.fdopen(fd, "w", encoding="utf-8") as stream:
            json.dump(to_json(value), stream, allow_nan=False, indent=2)
            stream.write("\n")
            stream.flush()
            os.fsync(stream.fileno())
        os.replace(tmp, path)
    finally:
        if os.path.exists(tmp):
            os.unlink(tmp)


def _h5py():
    try:
        import h5py
    except ImportError as err:
        raise TransportError("HDF5 array files need the h5py package", "runtime_failure") from err
    return h5py


def _dataset_names(key: str, complex_value: bool) -> dict:
    if complex_value:
        return {"real_dataset": f"/{key}_real", "imag_dataset": f"/{key}_imag"}
    return {"dataset": f"/{key}"}


def read_manifest(path, expected=None) -> dict:
    """A manifest checked against its schema without touching the arrays
    (wust_io.py:42-92): exact keys, object metadata, the required and only
    the known arrays, a sibling array file that exists, and per array its
    axes, units, dtype, shape (positive integers, one per axis) and dataset
    names."""
    path = Path(path).resolve(strict=True)
    doc = read_json(path)
    check_envelope(doc, expected)
    require_keys(doc, _MANIFEST_KEYS)
    if not isinstance(doc["metadata"], dict):
        raise TransportError("metadata must be an object")
    fields = ARRAY_FIELDS[doc["schema"]]
    require_keys(doc["arrays"], [k for k, f in fields.items() if not f.optional], fields)
    name = doc["arrays_file"]
    if not isinstance(name, str) or not name or Path(name).name != name:
        raise TransportError("arrays_file must be a sibling filename")
    data = (path.parent / name).resolve(strict=True)
    if data.parent != path.parent:
        raise TransportError("Array file must remain in the manifest directory")
    for key, spec in doc["arrays"].items():
        field = fields[key]
        complex_value = isinstance(spec, dict) and spec.get("dtype") in _COMPLEX
        require_keys(spec, {"shape", "dtype", "axes", "units"} | set(_dataset_names(key, complex_value)))
        units = doc["metadata"].get("data_units") if field.units == "data_units" else field.units
        if spec["axes"] not in field.axes or spec["units"] != units or spec["dtype"] not in field.dtypes:
            raise TransportError(f"Invalid axes/units/dtype for {key}")
        shape = spec["shape"]
        if (not isinstance(shape, list) or len(shape) != len(spec["axes"].split(","))
                or any(type(n) is not int or n < 1 for n in shape)):
            raise TransportError(f"Invalid shape for {key}")
        for dname, want in _dataset_names(key, complex_value).items():
            if spec[dname] != want:
                raise TransportError(f"Invalid dataset names for {key}")
    return doc


def read_artifact(path, expected=None):
    """(manifest, {name: array}) with every dataset checked against its
    descriptor's shape and storage type; booleans must hold only 0 and 1."""
    path = Path(path).resolve(strict=True)
    doc = read_manifest(path, expected)
    h5py = _h5py()
    arrays = {}
    with h5py.File(path.parent / doc["arrays_file"], "r") as handle:
        for key, spec in doc["arrays"].items():
            def load(dataset, dtype):
                obj = handle[dataset]
                if tuple(obj.shape) != tuple(spec["shape"]) or np.dtype(obj.dtype) != np.dtype(dtype):
                    raise TransportError(f"Dataset shape/dtype differs from manifest: {key}")
                return np.asarray(obj[...])

            if spec["dtype"] in _COMPLEX:
                part = "float32" if spec["dtype"] == "complex64" else "float64"
                value = load(spec["real_dataset"], part) + 1j * load(spec["imag_dataset"], part)
                value = value.astype(spec["dtype"])
            else:
                value = load(spec["dataset"], "uint8" if spec["dtype"] == "bool" else spec["dtype"])
                if spec["dtype"] == "bool":
                    if not np.isin(value, (0, 1)).all():
                        raise TransportError("Boolean dataset contains values other than 0/1")
                    value = value.astype(bool)
            arrays[key] = value
    return doc, arrays


def write_artifact(path, schema: str, metadata: dict, arrays: dict, axes: dict | None = None,
                   arrays_file: str | None = None) -> dict:
    """Write each array once into a new HDF5 file, then publish the manifest
    (wust_io.py:130-169).  ``axes`` overrides a field's first declared axis
    string; units come from the field table (``data_units`` from the
    metadata).  Returns the manifest."""
    path = Path(path).absolute()
    data = path.parent / arrays_file if arrays_file else path.with_suffix(".h5")
    if path.exists() or data.exists():
        raise FileExistsError(path)
    check_envelope({"schema": schema, "schema_version": PROTOCOL_VERSION})
    fields = ARRAY_FIELDS[schema]
    require_keys(arrays, [k for k, f in fields.items() if not f.optional], fields)
    h5py = _h5py()
    descriptors = {}
    with h5py.File(data, "x") as handle:
        for key, array in arrays.items():
            field = fields[key]
            value = np.asarray(array)
            ax = (axes or {}).get(key, field.axes[0])
            units = metadata.get("data_units") if field.units == "data_units" else field.units
            spec = {"shape": [int(n) for n in value.shape], "dtype": str(value.dtype), "axes": ax, "units": units}
            if len(spec["shape"]) != len(ax.split(",")) or spec["dtype"] not in field.dtypes:
                raise TransportError(f"Array {key} does not match its field ({spec['dtype']}, {ax})")
            spec.update(_dataset_names(key, np.iscomplexobj(value)))
            if np.iscomplexobj(value):
                handle.create_dataset(spec["real_dataset"], data=np.ascontiguousarray(value.real))
                handle.create_dataset(spec["imag_dataset"], data=np.ascontiguousarray(value.imag))
            else:
                handle.create_dataset(spec["dataset"],
                                      data=np.ascontiguousarray(value.astype(np.uint8) if value.dtype == bool else value))
            descriptors[key] = spec
    doc = {"schema": schema, "schema_version": PROTOCOL_VERSION, "metadata": to_json(metadata),
           "arrays_file": data.name, "arrays": descriptors}
    atomic_json(path, doc)
    return doc
