"""The strict restart contract (src/zhenmode/model/io/restart.py:17-227):
versioned, checksummed checkpoints that refuse every incompatible or damaged
file, written atomically, in the reference's file format."""
import copy
import hashlib
import json
from collections import namedtuple
from dataclasses import replace

import numpy as np
import pytest

from tests.golden_io import GOLDEN
from zhenmode_b200 import JaxStateG, restart, workloads

Params = namedtuple("Params", ["dt"])


def _setup(dtype="float64"):
    grid = workloads.build_grid(8, 8, 4, land_lat=80.0)
    shape = (8, 8, 4)
    zero = np.zeros(shape, dtype=dtype)
    surface = np.zeros((8, 8), dtype=dtype)
    state = JaxStateG(zero, zero.copy(), zero - 1.8, zero + 35.0, surface, surface + 0.5)
    contract = restart.make_restart_contract(
        grid, Params(60.0), dtype=dtype, forcing={"heat": np.zeros((8, 8))},
        controls={"calendar": "360_day"}, code_paths={"step": restart.__file__}, execution={"backend": "cpu"})
    return grid, state, contract


def _save(path, state, contract, step=12, **over):
    kw = dict(counters={"n_3d_snaps": 2}, cumulative={"salt": np.array([1.0, 2.0])},
              history={"days": np.array([0.0, 1.0]), "heat": np.array([3.0, 4.0])})
    kw.update(over)
    restart.save_restart(path, state, contract, step=step, **kw)


def _rewrite(path, edit):
    with np.load(path, allow_pickle=False) as saved:
        payload = {name: np.array(saved[name]) for name in saved.files}
    edit(payload)
    np.savez_compressed(path, **payload)


def _edit_metadata(payload, edit):
    metadata = json.loads(str(payload["metadata_json"]))
    edit(metadata)
    text = json.dumps(metadata, sort_keys=True, separators=(",", ":"), allow_nan=False)
    payload["metadata_json"] = np.asarray(text)
    payload["metadata_sha256"] = np.asarray(hashlib.sha256(text.encode()).hexdigest())


@pytest.mark.parametrize("dtype", ["float32", "float64"])
def test_round_trip_keeps_fields_dtype_time_counters_and_groups(tmp_path, dtype):
    _, state, contract = _setup(dtype)
    path = tmp_path / "ckpt.npz"
    _save(path, state, contract)
    got = restart.load_restart(path, contract)
    for name in state._fields:
        np.testing.assert_array_equal(got.state[name], getattr(state, name))
        assert got.state[name].dtype == np.dtype(dtype)
    assert got.step == 12 and got.elapsed_seconds == 720.0
    assert got.counters == {"n_3d_snaps": 2}
    np.testing.assert_array_equal(got.cumulative["salt"], [1.0, 2.0])
    np.testing.assert_array_equal(got.history["heat"], [3.0, 4.0])
    with np.load(path, allow_pickle=False) as raw:
        assert all(raw[name].dtype.kind != "O" for name in raw.files)


@pytest.mark.parametrize("field", ["grid", "effective_params", "forcing", "sources", "state_dtype",
                                   "execution", "controls", "dt_s"])
def test_incompatible_contract_is_refused(tmp_path, field):
    _, state, contract = _setup()
    path = tmp_path / "ckpt.npz"
    _save(path, state, contract)
    other = copy.deepcopy(contract)
    other[field] = "different"
    with pytest.raises(ValueError, match=f"contract mismatch: {field}"):
        restart.load_restart(path, other)


@pytest.mark.parametrize("field", ["lon", "z", "wet_mask_3d", "dx_2d"])
def test_changed_geometry_of_equal_size_is_refused(tmp_path, field):
    grid, state, contract = _setup()
    changed = np.array(getattr(grid, field), copy=True)
    changed.flat[-1] += 0.125
    other = restart.make_restart_contract(
        replace(grid, **{field: changed}), Params(60.0), dtype="float64", forcing={"heat": np.zeros((8, 8))},
        controls={"calendar": "360_day"}, code_paths={"step": restart.__file__}, execution={"backend": "cpu"})
    path = tmp_path / "ckpt.npz"
    _save(path, state, contract)
    with pytest.raises(ValueError, match="contract mismatch: grid"):
        restart.load_restart(path, other)


@pytest.mark.parametrize("step", [-1, 1.5, True, np.array([2])])
def test_steps_must_be_nonnegative_integers(tmp_path, step):
    _, state, contract = _setup()
    with pytest.raises(ValueError, match="nonnegative integer"):
        _save(tmp_path / "ckpt.npz", state, contract, step=step)


def test_unversioned_file_is_not_a_verified_restart(tmp_path):
    _, state, contract = _setup()
    path = tmp_path / "legacy.npz"
    np.savez(path, **{name: getattr(state, name) for name in state._fields if name != "ice"}, cur_step=12)
    with pytest.raises(ValueError, match="unversioned.*migration required"):
        restart.load_restart(path, contract)


@pytest.mark.parametrize("damage", ["missing_ice", "nonfinite", "shape", "dtype", "content", "history",
                                    "cumulative", "checksum", "extra"])
def test_damaged_payload_is_refused(tmp_path, damage):
    _, state, contract = _setup()
    path = tmp_path / "ckpt.npz"
    _save(path, state, contract)

    def edit(payload):
        if damage == "missing_ice":
            del payload["state__ice"]
        elif damage == "nonfinite":
            payload["state__T"][0, 0, 0] = np.nan
        elif damage == "shape":
            payload["state__eta"] = payload["state__eta"][:, :-1]
        elif damage == "dtype":
            payload["state__T"] = payload["state__T"].astype("float32")
        elif damage == "content":
            payload["state__T"][0, 0, 0] += 1.0
        elif damage == "history":
            payload["history__days"][1] += 1.0
        elif damage == "cumulative":
            payload["cumulative__salt"] *= 2.0
        elif damage == "checksum":
            payload["metadata_sha256"] = np.asarray("0" * 64)
        else:
            payload["unregistered"] = np.asarray(1.0)

    _rewrite(path, edit)
    with pytest.raises(ValueError):
        restart.load_restart(path, contract)


@pytest.mark.parametrize("damage", ["step", "time", "counter", "schema"])
def test_valid_checksum_does_not_hide_invalid_progress(tmp_path, damage):
    _, state, contract = _setup()
    path = tmp_path / "ckpt.npz"
    _save(path, state, contract)

    def edit(metadata):
        if damage == "step":
            metadata["step"] = 12.5
        elif damage == "time":
            metadata["elapsed_seconds"] += 0.1
        elif damage == "counter":
            metadata["counters"]["n_3d_snaps"] = -1
        else:
            metadata["schema_version"] += 1

    _rewrite(path, lambda payload: _edit_metadata(payload, edit))
    with pytest.raises(ValueError):
        restart.load_restart(path, contract)


@pytest.mark.parametrize("failure", ["write", "replace"])
def test_failed_save_keeps_previous_checkpoint(tmp_path, monkeypatch, failure):
    _, state, contract = _setup()
    path = tmp_path / "ckpt.npz"
    _save(path, state, contract)
    digest = restart.file_sha256(path)

    def fail(*args, **kwargs):
        raise OSError("injected storage failure")

    if failure == "write":
        monkeypatch.setattr(restart.np, "savez_compressed", fail)
    else:
        monkeypatch.setattr(restart.os, "replace", fail)
    with pytest.raises(OSError, match="injected"):
        _save(path, state, contract, step=13)
    monkeypatch.undo()
    assert restart.file_sha256(path) == digest
    assert restart.load_restart(path, contract).step == 12
    assert list(tmp_path.iterdir()) == [path]


def test_truncated_file_is_not_loaded(tmp_path):
    _, state, contract = _setup()
    path = tmp_path / "ckpt.npz"
    _save(path, state, contract)
    data = path.read_bytes()
    path.write_bytes(data[: len(data) // 2])
    with pytest.raises(Exception):
        restart.load_restart(path, contract)


@pytest.mark.parametrize("field", ["T", "ice"])
def test_invalid_state_cannot_overwrite_a_good_checkpoint(tmp_path, field):
    _, state, contract = _setup()
    path = tmp_path / "ckpt.npz"
    _save(path, state, contract)
    digest = restart.file_sha256(path)
    bad = np.array(getattr(state, field), copy=True)
    bad.flat[0] = np.inf
    with pytest.raises(ValueError):
        _save(path, state._replace(**{field: bad}), contract, step=13)
    assert restart.file_sha256(path) == digest


def _reference_inputs():
    data = dict(np.load(f"{GOLDEN}/restart_inputs.npz"))
    grid = workloads.build_grid(int(data["grid_nx"]), int(data["grid_ny"]), int(data["grid_nz"]),
                                land_lat=float(data["land_lat"]))
    pick = lambda prefix: {k[len(prefix):]: v for k, v in data.items() if k.startswith(prefix)}  # noqa: E731
    params = namedtuple("Params", ["dt", "nu_h", "polar_cap_rows"])(1800.0, 2.5e4, 2)
    contract = restart.make_restart_contract(grid, params, dtype="float32", forcing=pick("forcing_"),
                                             controls={"calendar": "360_day", "blend_days": 5.0}, code_paths={},
                                             execution={"backend": "cpu", "devices": 1})
    return contract, pick("state_"), pick("cumulative_"), pick("history_")


def test_reference_checkpoint_loads_and_is_written_identically(tmp_path):
    """A checkpoint from the reference's own save_restart (tests/golden/make_golden.py)
    loads here, and saving the same inputs here gives the same metadata and arrays."""
    contract, state, cumulative, history = _reference_inputs()
    ref_path = f"{GOLDEN}/restart_reference.npz"
    got = restart.load_restart(ref_path, contract)
    assert got.step == 96 and got.elapsed_seconds == 96 * 1800.0 and got.counters == {"n_snaps": 3}
    for name, value in state.items():
        np.testing.assert_array_equal(got.state[name], value)
    path = tmp_path / "ours.npz"
    restart.save_restart(path, state, contract, step=96, counters={"n_snaps": 3}, cumulative=cumulative,
                         history=history, outputs={"out/global.npz": "ab" * 32})
    with np.load(ref_path) as a, np.load(path) as b:
        assert sorted(a.files) == sorted(b.files)
        assert str(a["metadata_json"]) == str(b["metadata_json"])
        for name in a.files:
            np.testing.assert_array_equal(a[name], b[name])
