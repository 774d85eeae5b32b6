"""The allocation-free state check, zm_classify_state_noalloc, against the
solver's own monitor (zm_load_state + zm_advance(0) + zm_status).

The entry point is meant for callers that cannot call cudaMalloc (a runtime
whose memory pool owns the GPU, a check after a blow-up exhausted that pool,
a coupler on a fixed budget), so it keeps its scratch in a fixed array inside
the library.  Each state is checked twice in a row, because every call
reuses that array.  This file is collected last; it passes on its own and
after the other tests.
"""
import ctypes

import numpy as np
import pytest

from tests import gpu_util as gu
from zhenmode_b200 import _native, workloads

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    from oracle.params import init_state
    grid, physics, dt, kw, T, S = workloads.make_case("plain", 48, 24, 10, dtype="float32")
    gpu, p = gu.build_pair(grid, physics, dt, kw)
    return gpu.solver, gu.f32(init_state(p, T, S))


def _monitor_code(solver, fields, stream):
    sin = _native.ZmState(*[t.data_ptr() for t in fields])
    solver.check(solver.lib.zm_load_state(solver.handle, stream, ctypes.byref(sin)), "zm_load_state")
    solver.check(solver.lib.zm_advance(solver.handle, stream, 0), "zm_advance")
    code = ctypes.c_int32(-1)
    solver.check(solver.lib.zm_status(solver.handle, ctypes.byref(code)), "zm_status")
    return int(code.value)


def _noalloc(lib, fields, shape, stream, vlim=10.0, elim=15.0, inclusive=0):
    metrics = (ctypes.c_float * 4)()
    code = ctypes.c_int32(-1)
    rc = lib.zm_classify_state_noalloc(stream, *shape, *[ctypes.c_void_p(t.data_ptr()) for t in fields],
                                       vlim, elim, inclusive, metrics, ctypes.byref(code))
    return rc, int(code.value), list(metrics)


@pytest.mark.parametrize("edit", [
    lambda s: None,
    lambda s: s["T"].__setitem__((3, 4, 0), np.nan),
    lambda s: s["u"].__setitem__((5, 6, 2), 12.0),
    lambda s: s["v"].__setitem__((5, 6, 2), -10.5),
    lambda s: s["eta"].__setitem__((7, 8), 20.0),
    lambda s: (s["u"].__setitem__((1, 1, 1), 11.0), s["eta"].__setitem__((2, 2), 16.0)),
])
def test_noalloc_matches_monitor_twice(setup, edit):
    import torch
    solver, base = setup
    state = {k: np.array(v) for k, v in base.items()}
    edit(state)
    fields = gu.to_device(state)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    want = _monitor_code(solver, fields, stream)
    finite = all(np.isfinite(state[k]).all() for k in gu.FIELDS)
    for _ in range(2):
        rc, code, metrics = _noalloc(solver.lib, fields, solver.shape, stream)
        assert rc == _native.ZM_OK
        assert code == want
        assert metrics[3] == (1.0 if finite else 0.0)
        if finite:
            u32 = {k: np.asarray(state[k], dtype=np.float32) for k in gu.FIELDS}
            assert metrics[0] == np.abs(u32["u"]).max()
            assert metrics[1] == max(np.abs(u32["u"]).max(), np.abs(u32["v"]).max())
            assert metrics[2] == np.abs(u32["eta"]).max()


def test_noalloc_inclusive_limits(setup):
    import torch
    solver, base = setup
    state = {k: np.array(v) for k, v in base.items()}
    state["u"][0, 0, 0] = 10.0
    fields = gu.to_device(state)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert _noalloc(solver.lib, fields, solver.shape, stream, inclusive=0)[1] == 0
    assert _noalloc(solver.lib, fields, solver.shape, stream, inclusive=1)[1] == 3


def test_noalloc_rejects_fields_above_the_maximum(setup):
    import torch
    solver, base = setup
    fields = gu.to_device(base)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc, _, _ = _noalloc(solver.lib, fields, (4096, 4096, 16), stream)
    assert rc == _native.ZM_ERR_INVALID
