"""Device-side state monitor (runtime/monitor.py:20-30 codes) through the C
ABI: 0 accepted, 1 non-finite, 3 velocity above 10 m/s, 4 |eta| above 15 m,
with the reference's priority (non-finite > velocity > surface height).
Failures are injected into host-prepared states; nothing faults the GPU."""
import ctypes

import numpy as np
import pytest

from tests import gpu_util as gu
from zhenmode_b200 import _native, workloads

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def solver_state():
    from oracle.params import init_state
    grid, physics, dt, kw, T, S = workloads.make_case("plain", 48, 24, 10, dtype="float32")
    gpu, p = gu.build_pair(grid, physics, dt, kw)
    return gpu.solver, gu.f32(init_state(p, T, S))


def _code(solver, state):
    import torch
    fields = gu.to_device(state)
    sin = _native.ZmState(*[t.data_ptr() for t in fields])
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    solver.check(solver.lib.zm_load_state(solver.handle, stream, ctypes.byref(sin)), "zm_load_state")
    solver.check(solver.lib.zm_advance(solver.handle, stream, 0), "zm_advance")
    code = ctypes.c_int32(-1)
    solver.check(solver.lib.zm_status(solver.handle, ctypes.byref(code)), "zm_status")
    return int(code.value)


@pytest.mark.parametrize("edit,want", [
    (lambda s: None, 0),
    (lambda s: s["T"].__setitem__((3, 4, 0), np.nan), 1),
    (lambda s: s["u"].__setitem__((5, 6, 2), 12.0), 3),
    (lambda s: s["v"].__setitem__((5, 6, 2), -10.5), 3),
    (lambda s: s["eta"].__setitem__((7, 8), 20.0), 4),
    (lambda s: (s["u"].__setitem__((1, 1, 1), 11.0), s["eta"].__setitem__((2, 2), 16.0)), 3),
    (lambda s: (s["S"].__setitem__((1, 1, 1), np.inf), s["u"].__setitem__((2, 2, 2), 11.0)), 1),
])
def test_monitor_codes(solver_state, edit, want):
    solver, base = solver_state
    state = {k: np.array(v) for k, v in base.items()}
    edit(state)
    assert _code(solver, state) == want


def test_monitor_clears_between_calls(solver_state):
    solver, base = solver_state
    bad = {k: np.array(v) for k, v in base.items()}
    bad["u"][0, 0, 0] = np.nan
    assert _code(solver, bad) == 1
    assert _code(solver, base) == 0


def test_barrier_timeout_is_reported_and_context_survives(solver_state):
    """A grid barrier waiting for more blocks than exist gives up after its
    poll limit and reports ZM_ERR_TIMEOUT; the solver keeps working."""
    import torch
    solver, base = solver_state
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert solver.lib.zm_barrier_probe(solver.handle, stream, 8, 8, 1 << 20) == _native.ZM_OK
    assert solver.lib.zm_barrier_probe(solver.handle, stream, 8, 9, 20000) == _native.ZM_ERR_TIMEOUT
    assert _code(solver, base) == 0
