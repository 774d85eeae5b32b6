"""Strict restarts on the GPU (tests/runtime/test_restart_trajectory.py of the
reference): a run saved to a checkpoint after any step and resumed from it
ends bit for bit where the uninterrupted run ends, and n steps resident on the
device equal n calls of the jit-style ``step``."""
from collections import namedtuple

import numpy as np
import pytest

from zhenmode_b200 import JaxStateG, make_solver_global, restart, workloads

pytestmark = pytest.mark.gpu

FIELDS = ("u", "v", "T", "S", "eta", "ice")
Params = namedtuple("Params", ["dt"])


def _case(extra):
    grid, physics, dt, kw, T, S = workloads.make_case("plain", 48, 24, 10, dtype="float32")
    step, init, _ = make_solver_global(grid, physics, dt, **dict(kw, **extra))
    rng = np.random.default_rng(7)
    wet = np.asarray(grid.wet_mask_3d)
    st = init(T + 0.3 * rng.standard_normal(T.shape) * wet, S + 0.05 * rng.standard_normal(S.shape) * wet)
    st = step.advance(st, 4)  # a moving state
    contract = restart.make_restart_contract(grid, Params(dt), dtype="float32", forcing={},
                                             controls={"options": sorted(extra)}, code_paths={},
                                             execution={"backend": "cuda"})
    return step, st, contract


def _equal(a, b):
    import torch
    for k in FIELDS:
        x, y = getattr(a, k), getattr(b, k)
        x = x if isinstance(x, torch.Tensor) else torch.as_tensor(x, device="cuda")
        y = y if isinstance(y, torch.Tensor) else torch.as_tensor(y, device="cuda")
        assert torch.equal(x.cuda(), y.cuda()), k


@pytest.mark.parametrize("extra", [{}, {"project_adv_vel": True}, {"vertical_diffusion": "implicit"}])
def test_two_restarts_continue_bit_for_bit(tmp_path, extra):
    import torch
    step, st0, contract = _case(extra)
    continuous = step.advance(st0, 6)
    one_by_one = st0
    for _ in range(6):
        one_by_one = step(one_by_one)
    _equal(continuous, one_by_one)
    st = st0
    for n, chunk in enumerate((2, 3, 1)):
        st = step.advance(st, chunk)
        path = tmp_path / f"ckpt_{n}.npz"
        restart.save_restart(path, st, contract, step=n + 1, counters={}, cumulative={}, history={})
        saved = restart.load_restart(path, contract)
        st = JaxStateG(*[torch.as_tensor(saved.state[k], device="cuda") for k in FIELDS])
    _equal(continuous, st)
