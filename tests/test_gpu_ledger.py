"""The FP64 stage/source ledger of the GPU step (budget audit mode,
diagnostics/budgets.py:62-288) against the reference's own make_budget_step
on two steps with every legacy source on (sponge, eta relaxation, column
projection, bulk / coastal-bulk heat flux, SSS and coastal SST restoring,
brine rejection)."""
import numpy as np
import pytest

from tests import gpu_util as gu
from tests.golden_io import case_inputs, load
from zhenmode_b200 import JaxStateG, ledger, make_solver_global

pytestmark = pytest.mark.gpu

# Stage changes and sources are sums of per-cell float32 tracer increments:
# they are compared with the summed magnitudes of the changes they belong to.
# The magnitude sums themselves collect the float32 rounding of every
# increment without cancellation, hence their looser bound.
REL = 5e-4
REL_MAGNITUDE = 3e-3


def _setup():
    import torch
    data = load("ledger_48x24x10")
    grid, physics, dt, options, state = case_inputs(data)
    out = make_solver_global(grid, physics, dt, return_params=True, **dict(options, dtype="float32"))
    params = out[3]
    st = JaxStateG(*[torch.as_tensor(np.ascontiguousarray(state[k], dtype=np.float32), device="cuda")
                     for k in ("u", "v", "T", "S", "eta")],
                   torch.zeros((grid.nx, grid.ny), dtype=torch.float32, device="cuda"))
    return data, params, st


def _check(n, got, data):
    want = {k[len(f"ledger{n}_"):]: data[k] for k in data if k.startswith(f"ledger{n}_")}
    heat_salt_vol = np.maximum(np.asarray(want["change_scale"]), 1e-300)
    proc_scale = np.maximum(np.asarray(want["nonlinear_process_scale"]), 1e-300)
    for key, scale in (("observed_change", heat_salt_vol), ("stage_changes", heat_salt_vol),
                       ("source_inputs", heat_salt_vol), ("surface_displacement_tracer_change", heat_salt_vol),
                       ("change_scale", heat_salt_vol), ("nonlinear_process_changes", proc_scale),
                       ("nonlinear_process_scale", proc_scale), ("advection_boundary_changes", proc_scale)):
        g, w = np.asarray(got[key]), np.asarray(want[key])
        err = np.max(np.abs(g - w) / scale, axis=tuple(range(g.ndim - 1)) if g.ndim > 1 else None)
        bound = REL_MAGNITUDE if key.endswith("scale") else REL
        assert np.all(err <= bound), (n, key, err)
    # the projection norms: before to the float32 predictor's precision, after far below it
    nb, na = np.asarray(got["projection_transport_norm_squared"])
    wb, _ = want["projection_transport_norm_squared"]
    assert abs(nb - wb) <= 1e-3 * wb, (nb, wb)
    assert na <= 1e-9 * nb, (na, nb)


def test_ledger_matches_reference_budget_step():
    data, params, st = _setup()
    advance = ledger.make_budget_step(params)
    totals = ledger.empty_budget()
    for n in (1, 2):
        st, led = advance(st)
        got = {k: getattr(st, k).double().cpu().numpy() for k in gu.FIELDS}
        errs = gu.errors(got, {k: data[f"out{n}_{k}"] for k in gu.FIELDS})
        assert max(errs.values()) < 1e-5, (n, errs)
        assert set(led) == set(ledger.empty_budget())
        _check(n, led, data)
        # the stage decomposition telescopes on the device: it closes to rounding
        scale = np.asarray(led["change_scale"])
        assert np.all(np.abs(led["decomposition_residual"]) <= 1e-9 * np.maximum(scale, 1e-300)), led
        totals = ledger.accumulate_budget(totals, led)
    assert np.all(np.isfinite(totals["observed_change"]))


def test_ledger_step_equals_plain_step():
    """The audited step advances the state exactly like the graphed step."""
    import torch
    data, params, st = _setup()
    step = params.step
    plain = step(st)
    audited, _ = ledger.make_budget_step(params)(st)
    for k in ("u", "v", "T", "S", "eta"):
        assert torch.equal(getattr(plain, k), getattr(audited, k)), k
