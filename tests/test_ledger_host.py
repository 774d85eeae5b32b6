"""Host side of the budget audit: the ledger assembled from the raw device
sums has the reference's keys, shapes and residual identities
(diagnostics/budgets.py:234-262), checked on the reference's own ledger."""
import numpy as np

from tests.golden_io import load
from zhenmode_b200 import ledger


def _raw_from(led):
    raw = np.zeros(ledger.LEDGER_COUNT)
    raw[0:18] = np.asarray(led["stage_changes"]).ravel()
    raw[18:21] = led["change_scale"]
    raw[21:48] = np.asarray(led["source_inputs"]).ravel()
    raw[48:60] = np.asarray(led["nonlinear_process_changes"]).ravel()
    raw[60:63] = led["nonlinear_process_scale"]
    raw[63:66] = led["advection_boundary_changes"]
    raw[66:68] = led["projection_transport_norm_squared"]
    raw[68] = led["projection_relative_residual_max"]
    raw[69:72] = led["observed_change"]
    raw[72:75] = led["surface_displacement_tracer_change"]
    return raw


def test_ledger_assembly_reproduces_reference_ledger():
    data = load("ledger_48x24x10")
    for n in (1, 2):
        want = {k[len(f"ledger{n}_"):]: data[k] for k in data if k.startswith(f"ledger{n}_")}
        got = ledger.ledger_from_raw(_raw_from(want))
        assert set(got) == set(want) == set(ledger.empty_budget())
        for key, value in want.items():
            g = np.asarray(got[key], dtype=np.float64)
            assert g.shape == value.shape, key
            np.testing.assert_allclose(g, value, rtol=1e-12, atol=1e-12 * float(np.max(np.abs(value)) + 1), err_msg=key)


def test_accumulate_keeps_maxima_and_sums_the_rest():
    a, b = ledger.empty_budget(), ledger.empty_budget()
    a["observed_change"][:] = [1.0, 2.0, 3.0]
    b["observed_change"][:] = [0.5, 0.5, 0.5]
    a["projection_relative_residual_max"] = np.float64(0.3)
    b["projection_relative_residual_max"] = np.float64(0.1)
    t = ledger.accumulate_budget(ledger.accumulate_budget(ledger.empty_budget(), a), b)
    np.testing.assert_array_equal(t["observed_change"], [1.5, 2.5, 3.5])
    assert t["projection_relative_residual_max"] == 0.3
