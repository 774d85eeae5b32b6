"""Ensembles: one graph launch per step advancing members of uneven grid
sizes gives, member by member, exactly the states of advancing each member on
its own."""
import numpy as np
import pytest

from zhenmode_b200 import JaxStateG, make_solver_global, workloads
from zhenmode_b200.ensemble import Ensemble

pytestmark = pytest.mark.gpu


def _member(nx, ny, nz, seed, **extra):
    import torch
    grid, physics, dt, kw, T, S = workloads.make_case("plain", nx, ny, nz, dtype="float32")
    step, init, _ = make_solver_global(grid, physics, dt, **dict(kw, **extra))
    rng = np.random.default_rng(seed)
    wet = np.asarray(grid.wet_mask_3d)
    st = init(T + 0.05 * rng.standard_normal(T.shape) * wet, S)
    return step, st


def test_ensemble_matches_members_alone():
    import torch
    members = [_member(48, 24, 10, 1), _member(48, 24, 10, 2), _member(64, 32, 12, 3)]
    ens = Ensemble([m[0] for m in members])
    ens.load([m[1] for m in members])
    ens.advance(3)
    got = ens.store()
    assert ens.monitor_codes() == [0, 0, 0]
    assert ens.kernels_per_step > 0
    for (step, st), g in zip(members, got):
        want = step.advance(st, 3)
        for k in ("u", "v", "T", "S", "eta"):
            assert torch.equal(getattr(g, k), getattr(want, k)), k
    # the members' own steps in between force a recapture with the new parity
    ens.load([m[1] for m in members])
    ens.advance(2)
    ens.advance(1)
    again = ens.store()
    for a, b in zip(again, got):
        for k in ("u", "v", "T", "S", "eta"):
            assert torch.equal(getattr(a, k), getattr(b, k)), k


def test_ensemble_with_projection_matches_members_alone():
    """Two cooperative kernels per member (column projection, barotropic
    subcycle), chained across the members inside the one graph."""
    import torch
    members = [_member(48, 24, 10, 1, project_adv_vel=True),
               _member(64, 32, 12, 3, project_adv_vel=True, projection_preconditioner="jacobi")]
    ens = Ensemble([m[0] for m in members])
    ens.load([m[1] for m in members])
    ens.advance(2)
    got = ens.store()
    assert ens.monitor_codes() == [0, 0]
    for (step, st), g in zip(members, got):
        want = step.advance(st, 2)
        for k in ("u", "v", "T", "S", "eta"):
            assert torch.equal(getattr(g, k), getattr(want, k)), k


def test_handles_of_different_widths_coexist():
    """A narrow grid's handle created after a wide one leaves the wide one's
    kernels launchable (per-kernel launch limits are process-wide)."""
    import torch
    wide_step, wide_st = _member(96, 48, 10, 4)
    first = wide_step(wide_st)
    _member(24, 12, 6, 5)
    again = wide_step(wide_st)
    for k in ("u", "v", "T", "S", "eta"):
        assert torch.equal(getattr(first, k), getattr(again, k)), k


def test_autotuned_shapes_change_no_result():
    """The autotuner only picks among launch shapes with identical arithmetic."""
    import torch
    grid, physics, dt, kw, T, S = workloads.make_case("plain", 96, 48, 10, dtype="float32")
    plain, init, _ = make_solver_global(grid, physics, dt, **kw)
    tuned = make_solver_global(grid, physics, dt, autotune=True, **kw)[0]
    st = init(T, S)
    a = plain.advance(st, 2)
    b = tuned.advance(st, 2)
    halo, lines = tuned.solver.tuned_shapes()
    assert 3 <= halo <= 6 and lines in (1, 2, 4, 8)
    for k in ("u", "v", "T", "S", "eta"):
        assert torch.equal(getattr(a, k), getattr(b, k)), k
