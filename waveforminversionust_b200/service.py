"""The reference's runtime operations served by this library instead of MATLAB.

Runtime/python/wust_runtime.py validates a ``wust.request``, then runs
MATLAB's ``wust_run`` (Runtime/matlab/wust_run.m:1-74) in a supervised
process group with a hard deadline and publishes the result artifact.  This
module keeps that request/artifact contract (``transport``) and the same
supervision (a worker process in its own session, killed with its group at
the deadline; the run folder kept on failure for diagnosis), and executes
the operations with this library:

- ``ingest_frequency``: ``wust_prepare_observations`` (host);
- ``prepare``: RF -> canonical observations, the DTFT on the GPU
  (``wust_prepare``);
- ``reconstruct``: the frequency-continuation NCG loop with every oracle,
  curvature and update on the GPU (``wust_reconstruct``), in the precision
  profile the request's config names (``precision``, default
  ``tf32-refined``);
- ``simulate``: RF records of every transmitter from a sound-speed model,
  k-Wave's 2-D k-space method batched on the GPU (``wust_simulate``).

Command line, as the reference's:
``python -m waveforminversionust_b200.service describe`` and
``python -m waveforminversionust_b200.service run REQUEST --timeout-s S``.
"""
from __future__ import annotations

import argparse
import json
import os
import signal
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

from . import transport as T

RUNTIME_NAME = "WUST-B200"
RUNTIME_VERSION = "2.0.0-b200"
_PRECISIONS = ("c64", "c64-refined", "tf32-refined", "bf16-refined")


class RuntimeFailure(RuntimeError):
    def __init__(self, reason: str, message: str):
        super().__init__(message)
        self.reason = reason


def capabilities() -> dict:
    """What this runtime serves (the fields of wust_runtime.py:35-76, with
    the GPU profiles of this library)."""
    return {
        "schema": "wust.capabilities",
        "schema_version": T.PROTOCOL_VERSION,
        "runtime_name": RUNTIME_NAME,
        "runtime_version": RUNTIME_VERSION,
        "schemas": T.SCHEMAS,
        "operations": list(T.OPERATION_INPUTS),
        "input_schemas": {op: list(v) for op, v in T.OPERATION_INPUTS.items()},
        "sound_speed_reconstruction": {"supported": True, "dimensions": [2]},
        "attenuation_reconstruction": {"supported": False},
        "profiles": {"gpu": "gpu_complex64", **{f"gpu_{p}": p for p in _PRECISIONS}},
        "execution_platforms": ["Linux"],
        "iteration_unit": "frequency_schedule_update",
        "budgets": {"max_updates": True, "hard_timeout_s": True, "forward_call_cap": False,
                    "adjoint_call_cap": False, "update_rtol": False, "online_convergence": False},
        "source_scale": {"method": "per_tx_per_frequency_complex_least_squares", "minimum_fitting_receivers": 2,
                         "requires_water_reference": False, "requires_source_spectrum": False},
        "fourier_sign": -1,
    }


# ---------------------------------------------------------------------------
# the worker: one operation, inputs read from artifacts, result written


def _artifact_value(path, expected) -> dict:
    """An artifact as one dict: metadata, schema and arrays, plus the
    declared axes of a frequency input's pressure and mask
    (wust_read_artifact.m:15-67)."""
    doc, arrays = T.read_artifact(path, expected)
    value = dict(doc["metadata"])
    value.update(schema=doc["schema"], schema_version=doc["schema_version"])
    value.update(arrays)
    for key in ("pressure", "mask"):
        if key in doc["arrays"]:
            value[f"{key}_axes"] = doc["arrays"][key]["axes"]
    return value


def _observations(obs: dict):
    from .objective import Observations
    return Observations(obs["x_m"], obs["y_m"], obs["tx_index"], obs["rx_index"], obs["frequencies_hz"], obs["Y"],
                        obs["mask"])


def _measurements_artifact(obs: dict):
    arrays = {k: obs[k] for k in T.ARRAY_FIELDS["wust.measurements"]}
    arrays["tx_index"] = np.asarray(arrays["tx_index"], np.int64)
    arrays["rx_index"] = np.asarray(arrays["rx_index"], np.int64)
    arrays["Y"] = np.asarray(arrays["Y"], np.complex64)
    meta = {k: v for k, v in obs.items()
            if k not in arrays and k not in T.DERIVED_FIELDS and k not in ("schema", "schema_version")}
    return arrays, meta


def _environment(req: dict) -> dict:
    env = {"runtime_version": RUNTIME_VERSION, "platform": sys.platform, "python": sys.version.split()[0]}
    if req["operation"] in ("reconstruct", "prepare", "simulate"):
        import torch
        from . import _lib
        major, minor, patch = (_lib.C.c_int() for _ in range(3))
        _lib.load().wust_version(_lib.C.byref(major), _lib.C.byref(minor), _lib.C.byref(patch))
        props = torch.cuda.get_device_properties(torch.cuda.current_device())
        env.update(backend="gpu", gpu_device=props.name, compute_capability=f"{props.major}.{props.minor}",
                   library=_lib.LIB_PATH, library_version=f"{major.value}.{minor.value}.{patch.value}",
                   cuda_runtime=torch.version.cuda)
        if req["operation"] == "reconstruct":
            env["precision_profile"] = req["config"].get("precision", "tf32-refined")
    return env


def _reconstruction_artifact(result: dict, cfg: dict, obs: dict):
    arrays = {"c_mps": np.asarray(result["c_mps"], np.float64)}
    if "history_mps" in result:
        arrays["history_mps"] = np.asarray(result["history_mps"], np.float32)
    meta = {k: v for k, v in result.items() if k not in arrays and k not in ("schema", "schema_version")}
    schedule = [int(s) for s in result["executed_schedule"]]
    meta["executed_frequencies_hz"] = [float(obs["frequencies_hz"][s - 1]) for s in schedule]
    meta["canonical_frequencies_hz"] = np.asarray(obs["frequencies_hz"], np.float64)
    meta["observation_preparation"] = obs.get("preparation", {})
    meta["config"] = {k: v for k, v in cfg.items() if k != "update_mask"}
    return arrays, meta


def execute(req: dict) -> tuple[str, dict, dict]:
    """Run one validated request; returns (result schema, arrays, metadata)."""
    op = req["operation"]
    if op == "ingest_frequency":
        from .prepare import wust_prepare_observations
        obs = wust_prepare_observations(_artifact_value(req["input_manifest"], "wust.frequency_input"))
        return ("wust.measurements",) + _measurements_artifact(obs)
    if op == "prepare":
        from .prepare import wust_prepare
        rf = _artifact_value(req["input_manifest"], "wust.rf")
        cfg = dict(req["config"])
        units = rf.get("data_units")
        cfg["data_units"] = "Pa*s" if units == "Pa" else units          # wust_run.m:14-19
        cfg["measurement_provenance"] = rf.get("measurement_provenance")
        obs = wust_prepare(rf, cfg)
        return ("wust.measurements",) + _measurements_artifact(obs)
    if op == "reconstruct":
        from .prepare import wust_prepare_observations
        from .reconstruct import wust_reconstruct
        obs = wust_prepare_observations(
            _artifact_value(req["input_manifest"], ("wust.frequency_input", "wust.measurements")))
        initial = _artifact_value(req["initial_manifest"], "wust.initial_model")
        cfg = dict(req["config"])
        cfg["update_mask"] = initial["update_mask"]
        for key in ("frequency_schedule_hz", "max_updates", "save_history"):
            if key in req:
                cfg[key] = req[key]
        if "bounds_mps" in cfg:
            cfg["bounds_mps"] = np.asarray(cfg["bounds_mps"], np.float64)
        if cfg.get("precision", "tf32-refined") not in _PRECISIONS:
            from ._lib import WustError
            raise WustError(1, f"Unsupported precision profile {cfg.get('precision')!r}")
        result = wust_reconstruct(_observations(obs), np.asarray(initial["initial_mps"], np.float64), cfg)
        return ("wust.reconstruction",) + _reconstruction_artifact(result, cfg, obs)
    if op == "simulate":
        from .prepare import wust_geometry
        from .simulate import wust_simulate
        model = _artifact_value(req["input_manifest"], "wust.simulation_input")
        geo = wust_geometry(model["grid"], model["tx_xy_m"], model["rx_xy_m"])      # wust_run.m:33-39
        model.update(x_m=geo["x_m"], y_m=geo["y_m"], tx_index=geo["tx_index"], rx_index=geo["rx_index"])
        rf = wust_simulate(model, dict(req["config"]))
        arrays = {k: rf[k] for k in T.ARRAY_FIELDS["wust.rf"]}
        arrays["pressure"] = np.asarray(arrays["pressure"], np.float32)
        meta = {k: v for k, v in rf.items() if k not in arrays and k not in ("schema", "schema_version")}
        return "wust.rf", arrays, meta
    raise RuntimeFailure("runtime_failure", f"Operation {op!r} is not served by this runtime")


def _worker(internal_request: str) -> int:
    """Child process: execute the request written by ``run`` and write the
    result artifact into the run folder, or failure.json."""
    req = T.read_json(internal_request)
    out = Path(req["output_manifest"])
    started = time.perf_counter()
    try:
        schema, arrays, meta = execute(req)
        meta["runtime_wall_seconds"] = time.perf_counter() - started
        meta["environment"] = _environment(req)
        T.write_artifact(out, schema, meta, arrays, arrays_file="arrays.h5")
        return 0
    except Exception as err:  # noqa: BLE001 - reported through failure.json
        failure = {"schema": "wust.execution_failure", "schema_version": T.PROTOCOL_VERSION,
                   "identifier": getattr(err, "identifier", type(err).__name__), "message": str(err)}
        T.atomic_json(out.parent / "failure.json", failure)
        print(f"{failure['identifier']}: {failure['message']}", file=sys.stderr)
        return 1


# ---------------------------------------------------------------------------
# the launcher: validation, supervision, publication


def _kill_group(child: subprocess.Popen, grace_s: float = 0.5) -> None:
    """Stop the worker's process group (the worker leads it), then reap it."""
    for sig in (signal.SIGTERM, signal.SIGKILL):
        try:
            os.killpg(child.pid, sig)
        except ProcessLookupError:
            break
        deadline = time.monotonic() + grace_s
        while time.monotonic() < deadline:
            try:
                os.killpg(child.pid, 0)
            except ProcessLookupError:
                break
            child.poll()
            time.sleep(0.02)
    child.wait()


def _supervise(command, timeout_s: float, env=None) -> None:
    child = subprocess.Popen(command, start_new_session=True, stdout=sys.stderr, stderr=sys.stderr, env=env)
    try:
        code = child.wait(timeout=timeout_s)
    except subprocess.TimeoutExpired:
        _kill_group(child)
        raise
    except BaseException:
        _kill_group(child)
        raise
    if code:
        raise subprocess.CalledProcessError(code, command)


def run(request_path, timeout_s=None) -> dict:
    """Validate the request, execute it in a supervised worker and publish
    the result manifest at the request's output_manifest (wust_runtime.py:
    run and publish_runtime_output).  Returns the published manifest."""
    started = time.monotonic()
    req = T.validate_request(T.read_json(Path(request_path).resolve(strict=True)))
    if timeout_s is None:
        raise T.TransportError("An explicit timeout_s is required")
    T.check_number(timeout_s, "timeout_s")
    for key in ("input_manifest", "output_manifest", "initial_manifest"):
        if key in req and (not isinstance(req[key], str) or not Path(req[key]).is_absolute()):
            raise T.TransportError(f"{key} must be an absolute path")
    output = Path(req["output_manifest"])
    if output.exists() or output.is_symlink():
        raise FileExistsError(output)
    if not output.parent.is_dir():
        raise T.TransportError("Output parent must already exist")
    T.read_manifest(req["input_manifest"], T.OPERATION_INPUTS[req["operation"]])
    if req["operation"] == "reconstruct":
        T.read_manifest(req["initial_manifest"], "wust.initial_model")

    # the run folder keeps the request and any partial output on failure
    folder = Path(tempfile.mkdtemp(prefix=f"{output.stem}-run-", dir=output.parent))
    wire = dict(req, output_manifest=str(folder / "result.json"))
    if wire.get("frequency_schedule_hz") is None:
        wire.pop("frequency_schedule_hz", None)
    internal = folder / "request.json"
    T.atomic_json(internal, wire)
    remaining = timeout_s - (time.monotonic() - started)
    if remaining <= 0:
        raise RuntimeFailure("time_budget", "Timeout before the worker started")
    env = dict(os.environ)
    root = str(Path(__file__).resolve().parents[1])
    env["PYTHONPATH"] = root + (os.pathsep + env["PYTHONPATH"] if env.get("PYTHONPATH") else "")
    try:
        _supervise([sys.executable, "-m", "waveforminversionust_b200.service", "_worker", str(internal)],
                   remaining, env)
    except subprocess.TimeoutExpired as err:
        raise RuntimeFailure("time_budget", "Deadline expired; worker process group terminated") from err
    except (OSError, subprocess.CalledProcessError) as err:
        failure = folder / "failure.json"
        detail = T.read_json(failure) if failure.exists() else {}
        reason = "numerical_failure" if detail.get("identifier") == "WUST:NumericalFailure" else "runtime_failure"
        raise RuntimeFailure(reason, detail.get("message", str(err))) from err
    result_path = Path(wire["output_manifest"])
    if not result_path.is_file():
        raise RuntimeFailure("incomplete_output", "Worker exited without completed output")
    result = T.read_manifest(result_path, T.OPERATION_OUTPUT[req["operation"]])
    result["metadata"].update(runtime_version=RUNTIME_VERSION, request_timeout_s=timeout_s,
                              process_wall_seconds=time.monotonic() - started)
    if time.monotonic() - started >= timeout_s:
        raise RuntimeFailure("time_budget", "Deadline expired before final publication")
    # publication: the arrays move next to the output, then the manifest
    # appears (the success index), then the run folder's copy goes
    destination = output.parent / f"{folder.name}.h5"
    os.replace(folder / result["arrays_file"], destination)
    result["arrays_file"] = destination.name
    T.atomic_json(output, result)
    result_path.unlink()
    return result


def main(argv=None) -> None:
    parser = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    commands = parser.add_subparsers(dest="command", required=True)
    commands.add_parser("describe")
    run_parser = commands.add_parser("run")
    run_parser.add_argument("request")
    run_parser.add_argument("--timeout-s", type=float, required=True)
    worker = commands.add_parser("_worker")
    worker.add_argument("request")
    args = parser.parse_args(argv)
    if args.command == "_worker":
        raise SystemExit(_worker(args.request))
    try:
        result = capabilities() if args.command == "describe" else run(args.request, args.timeout_s)
        print(json.dumps(T.to_json(result), allow_nan=False))
    except (OSError, ValueError, RuntimeError) as err:
        print(json.dumps({"schema": "wust.execution_failure", "schema_version": T.PROTOCOL_VERSION,
                          "reason": getattr(err, "reason", "incompatible_request"), "message": str(err)}),
              file=sys.stderr)
        raise SystemExit(1) from err


if __name__ == "__main__":
    main()
