"""The drop-in boundary as the reference runtime uses it
(src/zhenmode/model/runtime/run.py:49-131):

* ``make_solver_global(..., return_params=True)`` returns a params object
  whose fields are what the run reporting, the output provenance and the
  restart contract read (runtime/reporting.py:22-25, io/output.py:89-96,
  io/restart.py:56-75), and which zhenmode_b200.ledger.make_budget_step takes
  the way run.py:113-127 calls RunServices.make_budget_step;
* ``terms_fn`` (factory.py:762-764) gives the reference's tracer-term stack,
  checked against the reference's own ``_tracer_terms`` output
  (tests/golden/terms_48x24x10.npz).
"""
import numbers

import numpy as np
import pytest

from tests import gpu_util as gu
from tests.golden_io import grid_from, load
from zhenmode_b200 import JaxStateG, ledger, make_solver_global, workloads
from zhenmode_b200.solver import B200Params

pytestmark = pytest.mark.gpu

TERM_TOL = 1e-5


def _terms_case():
    data = load("terms_48x24x10")
    grid = grid_from(data)
    wm = np.asarray(grid.wet_mask)
    kw = dict(workloads.PLAIN_OPTIONS)
    kw.update(forcing=workloads.wind_forcing(grid), dt_bt=75.0, dtype="float32",
              coastal_kappa_h_mask=wm, coastal_kappa_h=float(data["coastal_kappa_h"]),
              coastal_kappa_v_mask=wm, coastal_kappa_v=float(data["coastal_kappa_v"]))
    state = {k: data["in_" + k] for k in ("u", "v", "T", "S", "eta")}
    return data, grid, kw, state


def test_terms_fn_matches_reference_terms():
    data, grid, kw, state = _terms_case()
    out = make_solver_global(grid, workloads.PLAIN_PHYSICS, 1800.0, return_params=True, **kw)
    terms_fn = out[4]
    got_dev = terms_fn(JaxStateG(*gu.to_device(state), 0.0))
    got_host = terms_fn(JaxStateG(*[np.asarray(state[k], np.float32) for k in gu.FIELDS], 0.0))
    want = data["terms"]
    assert tuple(got_dev.shape) == want.shape and got_host.shape == want.shape
    assert np.array_equal(got_dev.cpu().numpy(), got_host)
    for n, name in enumerate(("adv", "diff_h", "diff_v", "conv", "gm", "redi")):
        if np.abs(want[n]).max() == 0:
            assert np.abs(got_host[n]).max() == 0, name
        else:
            err = gu.rel_l2(got_host[n], want[n])
            assert err < TERM_TOL, (name, err)


def _fingerprintable(value):
    """The value kinds the reference's restart fingerprint accepts
    (io/restart.py:34-51): numbers, strings, flags, None, finite arrays."""
    if value is None or isinstance(value, (str, bool, numbers.Number)):
        return True
    a = np.asarray(value)
    return a.dtype.kind in "biuf" and bool(np.isfinite(a).all())


def test_params_serve_the_reference_runtime():
    grid, physics, dt, kw, T, S = workloads.make_case("plain", 48, 24, 10, dtype="float32")
    step, init, _, params, terms_fn = make_solver_global(grid, physics, dt, return_params=True, **kw)
    assert isinstance(params, B200Params)
    # runtime/reporting.py:22-25 and io/output.py:89-96
    assert params.n_subcyc == round(dt / 75.0) and params.nu_nsub == params.n_subcyc
    assert params.conv_nsub >= 1 and params.adv_nsub >= 1 and params.use_scan == kw.get("use_scan", False)
    assert params.dt_bt == pytest.approx(dt / params.n_subcyc)
    assert params.wet_mask_z.shape == (48, 24, 10) and params.wet_mask_z.dtype == np.float32
    assert params.projection_niter_source == "default"
    assert all(_fingerprintable(v) for v in params._asdict().values())
    # run.py:113-121: the audited step beside the ordinary one
    audited = ledger.make_budget_step(params)
    st = step.advance(init(T, S), 2)
    plain = step(st)
    checked, budget = audited(st)
    for k in gu.FIELDS:
        assert np.array_equal(getattr(plain, k).cpu().numpy(), getattr(checked, k).cpu().numpy()), k
    assert set(budget) == set(ledger.empty_budget())
    assert np.all(np.isfinite(budget["observed_change"]))


def test_params_serve_the_dynamic_runtime_path():
    """run.py:123-127: audited_step(state, (tx, ty, heat), T_atm_3d) beside
    step_dyn with the same forcing."""
    grid, physics, dt, kw, T, S = workloads.make_case("plain", 48, 24, 10, dtype="float32")
    step, init, _, params, _, step_dyn = make_solver_global(grid, physics, dt, return_params=True,
                                                            dynamic_forcing=True, **kw)
    audited = ledger.make_budget_step(params)
    st = step.advance(init(T, S), 1)
    lat = np.radians(np.asarray(grid.lat))
    tx = np.broadcast_to((0.12 * np.sin(2 * lat) * np.cos(lat))[None, :], (48, 24)).astype(np.float32)
    ty = np.zeros((48, 24), np.float32)
    q = np.broadcast_to((50.0 * np.cos(lat))[None, :], (48, 24)).astype(np.float32)
    dyn = step_dyn(st, tx, ty, q)
    checked, budget = audited(st, (tx, ty, q), None)
    for k in gu.FIELDS:
        assert np.array_equal(getattr(dyn, k).cpu().numpy(), getattr(checked, k).cpu().numpy()), k
    assert abs(budget["source_inputs"][0, 0]) > 0  # the prescribed heat flux entered the ledger
