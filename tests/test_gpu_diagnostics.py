"""The diagnostics closure (rho, pressure, w) and the float64 budget snapshot
on the GPU, through the C ABI, against golden values of the reference's own
code (tests/golden/diagnostics_48x24x10.npz) and the float64 oracle."""
import numpy as np
import pytest

from oracle import budgets as obudgets
from tests.golden_io import grid_from, load, rel_l2
from zhenmode_b200 import JaxStateG, compute_budget_diagnostics, make_solver_global, workloads

pytestmark = pytest.mark.gpu

DIAG_TOL = 1e-5       # float32 fields, relative L2
BUDGET_TOL = 1e-12    # float64 sums of the same float32 inputs, relative


@pytest.fixture(scope="module")
def case():
    data = load("diagnostics_48x24x10")
    grid = grid_from(data)
    lat = np.radians(np.asarray(grid.lat))
    tau_x = np.broadcast_to((0.1 * np.sin(2 * lat) * np.cos(lat))[None, :], (grid.nx, grid.ny)).copy()
    zeros = np.zeros((grid.nx, grid.ny))
    kw = dict(workloads.PLAIN_OPTIONS)
    kw.update(forcing=(tau_x, zeros, zeros.copy()), dt_bt=75.0, dtype="float32")
    step, _, diagnostics = make_solver_global(grid, workloads.PLAIN_PHYSICS, 1800.0, **kw)
    return data, grid, step, diagnostics


def _state(data, device):
    import torch
    arrs = [np.asarray(data["in_" + k], dtype=np.float32) for k in ("u", "v", "T", "S", "eta")]
    if device:
        arrs = [torch.as_tensor(a, device="cuda") for a in arrs]
    return JaxStateG(*arrs, None)


@pytest.mark.parametrize("device", [True, False])
def test_diagnostics_match_reference(case, device):
    data, _, _, diagnostics = case
    st = _state(data, device)
    rho, pres, w = diagnostics(st)
    _, pres_sp, _ = diagnostics(st, surface_pressure_pa=data["surface_pressure_pa"])
    got = dict(rho=rho, pressure=pres, w=w, pressure_sp=pres_sp)
    for name, arr in got.items():
        arr = arr.cpu().numpy() if device else arr
        err = rel_l2(arr, data[name])
        assert err < DIAG_TOL, (name, err)


def test_budgets_match_reference(case):
    data, _, step, _ = case
    st = _state(data, True)
    b = compute_budget_diagnostics(st, solver=step)
    names = [str(n) for n in data["budget_names"]]
    for name, want in zip(names, data["budget_values"]):
        got = getattr(b, name)
        assert abs(got - want) <= BUDGET_TOL * abs(want), (name, got, want)
    again = step.budget_diagnostics(st)
    assert again == b   # fixed summation order: bit-identical


def test_budgets_match_oracle_at_production_depth():
    """180x90x50 with the 0.5-degree option set and a perturbed state."""
    import torch
    grid, physics, dt, kw, T, S = workloads.make_case("plain", 180, 90, 50, dtype="float32")
    step = make_solver_global(grid, physics, dt, **kw)[0]
    rng = np.random.default_rng(3)
    T32 = (T + 0.3 * rng.standard_normal(T.shape)).astype(np.float32)
    S32 = (S + 0.05 * rng.standard_normal(S.shape)).astype(np.float32)
    zeros = np.zeros(T.shape, np.float32)
    st = JaxStateG(*[torch.as_tensor(a, device="cuda") for a in (zeros, zeros, T32, S32)],
                   torch.zeros(T.shape[:2], device="cuda"), None)
    got = step.budget_diagnostics(st).as_dict()
    want = obudgets.budget_diagnostics(T32, S32, grid.dx_2d, grid.dy, grid.z, grid.wet_mask, grid.wet_mask_3d)
    for name in obudgets.FIELDS:
        assert abs(got[name] - want[name]) <= BUDGET_TOL * abs(want[name]), (name, got[name], want[name])
