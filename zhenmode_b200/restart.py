"""Strict restarts of the B200 step (the checkpoint contract of
src/zhenmode/model/io/restart.py:17-227).

A checkpoint is one ``.npz`` archive.  Its arrays sit under
``"<group>__<name>"`` keys for the three groups ``state`` (u, v, T, S, eta,
ice), ``cumulative`` and ``history``; ``metadata_json`` holds the canonical
JSON (sorted keys, compact separators, no NaN) of the schema version, the
frozen contract, step, elapsed seconds (= step * dt), integer counters, output
digests and a descriptor of every array (shape, dtype string, SHA-256 of the
C-order bytes), and ``metadata_sha256`` its digest.  The layout is the
reference's, so a checkpoint written by either code loads in the other when
the contracts are equal.

Loading verifies everything before any state is handed back: the metadata
checksum, the schema, the contract (every mismatching top-level key is
named), step * dt, each array's descriptor, and that the archive holds no
other array.  Saving writes a temporary file in the same directory, fsyncs it
and renames it over the target, so a failed save leaves the previous
checkpoint as it was.

The B200 step is restart-exact: a state saved after any step and loaded again
continues bit for bit like the uninterrupted run (the device state after each
step is exactly the one that loading the step's output gives).
"""
from __future__ import annotations

import hashlib
import json
import os
import tempfile
from contextlib import contextmanager
from dataclasses import dataclass, fields, is_dataclass
from pathlib import Path, PurePosixPath

import numpy as np

SCHEMA_VERSION = 1
STATE_FIELDS = ("u", "v", "T", "S", "eta", "ice")
GROUPS = ("state", "cumulative", "history")
_HEX = frozenset("0123456789abcdef")


def _canonical_json(value):
    return json.dumps(value, sort_keys=True, separators=(",", ":"), allow_nan=False)


def _host_array(value):
    """numpy view of an array-like, torch tensors included (copied to the host)."""
    if hasattr(value, "detach") and hasattr(value, "cpu"):
        value = value.detach().cpu().numpy()
    return np.asarray(value)


def describe(value):
    """Shape, dtype string and SHA-256 of the C-order bytes of a finite real array."""
    array = _host_array(value)
    if array.dtype.kind not in "biuf" or not np.isfinite(array).all():
        raise ValueError("restart arrays must be finite real numeric arrays without pickle")
    digest = hashlib.sha256(array.tobytes(order="C")).hexdigest()
    return {"shape": list(array.shape), "dtype": array.dtype.str, "sha256": digest}


def fingerprint(value):
    """JSON-able identity of effective values: dataclasses and named tuples by
    field, mappings by (string) key, sequences in order, scalars as themselves,
    arrays by their descriptor."""
    if is_dataclass(value) and not isinstance(value, type):
        return {f.name: fingerprint(getattr(value, f.name)) for f in fields(value)}
    if hasattr(value, "_asdict"):
        return fingerprint(value._asdict())
    if isinstance(value, dict):
        if not all(isinstance(key, str) for key in value):
            raise ValueError("restart mappings require string keys")
        return {key: fingerprint(item) for key, item in value.items()}
    if isinstance(value, (list, tuple)):
        return [fingerprint(item) for item in value]
    if value is None or isinstance(value, (bool, int, str)):
        return value
    if isinstance(value, float):
        if not np.isfinite(value):
            raise ValueError("restart contract contains a nonfinite scalar")
        return value
    return describe(value)


def file_sha256(path, chunk=1 << 20):
    h = hashlib.sha256()
    with open(path, "rb") as stream:
        for block in iter(lambda: stream.read(chunk), b""):
            h.update(block)
    return h.hexdigest()


def make_restart_contract(grid, params, *, dtype, forcing, controls, code_paths, execution):
    """Freeze what a continuation must share: state shapes and dtype, dt, the
    grid, the effective parameters, forcing, run controls, source digests and
    the execution environment."""
    nx, ny, nz = int(grid.nx), int(grid.ny), int(grid.nz)
    state_dtype = np.dtype(dtype)
    if state_dtype.name not in ("float32", "float64"):
        raise ValueError("restart compute dtype must be float32 or float64")
    dt = float(params.dt)
    if not (np.isfinite(dt) and dt > 0.0):
        raise ValueError("restart dt must be finite and positive")
    shapes = {name: ([nx, ny] if name in ("eta", "ice") else [nx, ny, nz]) for name in STATE_FIELDS}
    return {"schema_version": SCHEMA_VERSION,
            "state_family": "FD_point_samples_linear_free_surface",
            "state_shapes": shapes,
            "state_dtype": state_dtype.str,
            "dt_s": dt,
            "grid": fingerprint(grid),
            "effective_params": fingerprint(params),
            "forcing": fingerprint(forcing),
            "controls": fingerprint(controls),
            "sources": {name: file_sha256(path) for name, path in code_paths.items()},
            "execution": fingerprint(execution)}


def _count(value, what):
    array = np.asarray(value)
    if array.shape != () or array.dtype.kind not in "iu" or int(array) < 0:
        raise ValueError(f"restart {what} must be a nonnegative integer scalar")
    return int(array)


def _arrays(mapping, group):
    if not isinstance(mapping, dict) or not all(isinstance(k, str) and k and "__" not in k for k in mapping):
        raise ValueError(f"restart {group} requires nonempty string array names without '__'")
    out = {name: np.array(_host_array(value), copy=True) for name, value in mapping.items()}
    for array in out.values():
        describe(array)
    return out


def _state_arrays(state, contract):
    if hasattr(state, "_asdict"):
        state = state._asdict()
    if set(state) != set(STATE_FIELDS):
        raise ValueError("restart must contain all six state fields including ice")
    arrays = _arrays(state, "state")
    for name, array in arrays.items():
        if list(array.shape) != contract["state_shapes"][name]:
            raise ValueError(f"restart {name} shape differs from the frozen grid")
        if array.dtype.str != contract["state_dtype"]:
            raise ValueError(f"restart {name} dtype differs from the frozen compute dtype")
    return arrays


def _check_outputs(outputs):
    if not isinstance(outputs, dict):
        raise ValueError("restart outputs must be a mapping")
    for name, digest in outputs.items():
        safe = (isinstance(name, str) and name and "\\" not in name and ":" not in name
                and not PurePosixPath(name).is_absolute() and ".." not in PurePosixPath(name).parts)
        if not (safe and isinstance(digest, str) and len(digest) == 64 and set(digest) <= _HEX):
            raise ValueError("restart output paths/hashes must be safe relative paths and SHA256")


@dataclass(frozen=True)
class RestartRecord:
    state: dict
    step: int
    elapsed_seconds: float
    counters: dict
    cumulative: dict
    history: dict
    outputs: dict


@contextmanager
def atomic_archive(path, *, replace=False):
    """Write through a same-directory temporary file, fsync, then publish:
    ``replace=True`` renames over the target, otherwise a hard link refuses an
    existing one.  The temporary file never outlives the block."""
    path = Path(path)
    tmp = None
    try:
        with tempfile.NamedTemporaryFile(dir=path.parent, prefix=f".{path.name}.", suffix=".tmp",
                                         delete=False) as stream:
            tmp = Path(stream.name)
            yield stream
            stream.flush()
            os.fsync(stream.fileno())
        if replace:
            os.replace(tmp, path)
        else:
            os.link(tmp, path)
    finally:
        if tmp is not None and tmp.exists():
            tmp.unlink()


def save_restart(path, state, contract, *, step, counters, cumulative, history, outputs=None):
    """Checkpoint ``state`` (a JaxStateG or mapping of the six fields, host or
    device arrays) after ``step`` steps; replaces ``path`` atomically."""
    if contract.get("schema_version") != SCHEMA_VERSION:
        raise ValueError("unsupported restart contract version")
    step = _count(step, "step")
    counters = {name: _count(value, name) for name, value in counters.items()}
    groups = {"state": _state_arrays(state, contract),
              "cumulative": _arrays(cumulative, "cumulative"),
              "history": _arrays(history, "history")}
    outputs = dict(outputs or {})
    _check_outputs(outputs)
    elapsed = step * contract["dt_s"]
    if not np.isfinite(elapsed):
        raise ValueError("restart elapsed time is nonfinite")
    metadata = {"schema_version": SCHEMA_VERSION, "contract": contract, "step": step,
                "elapsed_seconds": elapsed, "counters": counters, "outputs": outputs,
                "arrays": {g: {n: describe(a) for n, a in arrays.items()} for g, arrays in groups.items()}}
    text = _canonical_json(metadata)
    payload = {f"{g}__{n}": a for g, arrays in groups.items() for n, a in arrays.items()}
    payload["metadata_json"] = np.asarray(text)
    payload["metadata_sha256"] = np.asarray(hashlib.sha256(text.encode()).hexdigest())
    with atomic_archive(path, replace=True) as stream:
        np.savez_compressed(stream, **payload)


def load_restart(path, expected_contract):
    """Verify and read a checkpoint; raises ValueError on any mismatch before
    returning state."""
    with np.load(path, allow_pickle=False) as saved:
        if "metadata_json" not in saved or "metadata_sha256" not in saved:
            raise ValueError("unversioned checkpoint is not a verified restart; migration required")
        text_arr, digest_arr = saved["metadata_json"], saved["metadata_sha256"]
        if text_arr.shape != () or text_arr.dtype.kind != "U" or digest_arr.shape != ():
            raise ValueError("restart metadata must be scalar JSON and checksum")
        text = str(text_arr)
        if hashlib.sha256(text.encode()).hexdigest() != str(digest_arr):
            raise ValueError("restart metadata checksum mismatch")
        metadata = json.loads(text)
        if metadata.get("schema_version") != SCHEMA_VERSION:
            raise ValueError("unsupported restart schema version")
        frozen = metadata["contract"]
        if _canonical_json(frozen) != _canonical_json(expected_contract):
            keys = [key for key in expected_contract if frozen.get(key) != expected_contract[key]]
            raise ValueError(f"restart contract mismatch: {', '.join(keys)}")
        step = _count(metadata["step"], "step")
        elapsed = step * expected_contract["dt_s"]
        if not np.isfinite(elapsed) or metadata["elapsed_seconds"] != elapsed:
            raise ValueError("restart absolute time differs from step * frozen dt")
        counters = {name: _count(value, name) for name, value in metadata["counters"].items()}
        _check_outputs(metadata["outputs"])
        if set(metadata["arrays"]) != set(GROUPS):
            raise ValueError("restart array groups mismatch")
        expected_keys = {"metadata_json", "metadata_sha256"}
        groups = {}
        for group, descriptors in metadata["arrays"].items():
            groups[group] = {}
            for name, descriptor in descriptors.items():
                key = f"{group}__{name}"
                expected_keys.add(key)
                if key not in saved:
                    raise ValueError(f"restart missing array {key}")
                value = np.array(saved[key], copy=True)
                if describe(value) != descriptor:
                    raise ValueError(f"restart array content/shape/dtype mismatch: {key}")
                groups[group][name] = value
            _arrays(groups[group], group)
        if set(saved.files) != expected_keys:
            raise ValueError("restart contains unexpected arrays")
    state = _state_arrays(groups["state"], expected_contract)
    return RestartRecord(state, step, elapsed, counters, groups["cumulative"], groups["history"],
                         metadata["outputs"])
