"""The allocation-free state check, zm_classify_state_noalloc, against the
solver's own monitor (zm_load_state + zm_advance(0) + zm_status) and the
NumPy maxima of the same float32 arrays.

The entry point is meant for callers that cannot call cudaMalloc (a runtime
whose memory pool owns the GPU, a check after a blow-up exhausted that pool,
a coupler on a fixed budget), so it keeps its scratch in a fixed array inside
the library.  Each state is checked twice in a row, because every call
reuses that array.  The 48x24x10 state is one block of the kernel; the
200x100x20 state is seven, so the per-block partials, the last-block fold and
the counter reset run, with the planted values in the last blocks.  This file
is collected last; it passes on its own and after the other tests.
"""
import ctypes

import numpy as np
import pytest

from tests import gpu_util as gu
from zhenmode_b200 import _native, workloads

pytestmark = pytest.mark.gpu

CHUNK = 65536  # 3-D points per block of the kernel


def _case(nx, ny, nz):
    from oracle.params import init_state
    grid, physics, dt, kw, T, S = workloads.make_case("plain", nx, ny, nz, dtype="float32")
    gpu, p = gu.build_pair(grid, physics, dt, kw)
    st = gu.f32(init_state(p, T, S))
    rng = np.random.default_rng(11)
    wm = p.wet_mask_z
    st["u"] = (0.3 * rng.standard_normal(wm.shape) * wm).astype(np.float32).astype(np.float64)
    st["v"] = (0.3 * rng.standard_normal(wm.shape) * wm).astype(np.float32).astype(np.float64)
    st["eta"] = (0.5 * rng.standard_normal(wm.shape[:2]) * p.wet_mask).astype(np.float32).astype(np.float64)
    return gpu.solver, st


@pytest.fixture(scope="module")
def small():
    return _case(48, 24, 10)


@pytest.fixture(scope="module")
def multi():
    return _case(200, 100, 20)


def _monitor_code(solver, fields, stream):
    sin = _native.ZmState(*[t.data_ptr() for t in fields])
    solver.check(solver.lib.zm_load_state(solver.handle, stream, ctypes.byref(sin)), "zm_load_state")
    solver.check(solver.lib.zm_advance(solver.handle, stream, 0), "zm_advance")
    code = ctypes.c_int32(-1)
    solver.check(solver.lib.zm_status(solver.handle, ctypes.byref(code)), "zm_status")
    return int(code.value)


def _noalloc(lib, fields, shape, stream, ice=None, vlim=10.0, elim=15.0, inclusive=0):
    metrics = (ctypes.c_float * 4)()
    code = ctypes.c_int32(-1)
    ptr = ctypes.c_void_p(ice.data_ptr()) if ice is not None else ctypes.c_void_p(None)
    rc = lib.zm_classify_state_noalloc(stream, *shape, *[ctypes.c_void_p(t.data_ptr()) for t in fields], ptr,
                                       vlim, elim, inclusive, metrics, ctypes.byref(code))
    return rc, int(code.value), list(metrics)


def _jnp_max(a):
    """jnp.max(jnp.abs(a)) of float32 values: NaN if any NaN."""
    a = np.abs(np.asarray(a, dtype=np.float32))
    return float("nan") if np.isnan(a).any() else float(a.max())


def _same(x, y):
    return (np.isnan(x) and np.isnan(y)) or x == y


def _check(solver, state, ice=None):
    import torch
    fields = gu.to_device(state)
    ice_t = torch.as_tensor(np.ascontiguousarray(ice, dtype=np.float32), device="cuda") if ice is not None else None
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    want = _monitor_code(solver, fields, stream)
    finite = all(np.isfinite(np.asarray(state[k], np.float32)).all() for k in gu.FIELDS)
    if ice is not None:
        finite = finite and bool(np.isfinite(ice).all())
        want = 1 if not finite else want
    mu, mv, me = _jnp_max(state["u"]), _jnp_max(state["v"]), _jnp_max(state["eta"])
    mvel = float("nan") if np.isnan(mu) or np.isnan(mv) else max(mu, mv)
    for _ in range(2):
        rc, code, metrics = _noalloc(solver.lib, fields, solver.shape, stream, ice=ice_t)
        assert rc == _native.ZM_OK
        assert code == want
        assert metrics[3] == (1.0 if finite else 0.0)
        assert _same(metrics[0], mu) and _same(metrics[1], mvel) and _same(metrics[2], me), (metrics, mu, mvel, me)


@pytest.mark.parametrize("edit", [
    lambda s: None,
    lambda s: s["T"].__setitem__((3, 4, 0), np.nan),
    lambda s: s["u"].__setitem__((5, 6, 2), 12.0),
    lambda s: s["v"].__setitem__((5, 6, 2), -10.5),
    lambda s: s["eta"].__setitem__((7, 8), 20.0),
    lambda s: (s["u"].__setitem__((1, 1, 1), 11.0), s["eta"].__setitem__((2, 2), 16.0)),
])
def test_noalloc_matches_monitor_twice(small, edit):
    solver, base = small
    state = {k: np.array(v) for k, v in base.items()}
    edit(state)
    _check(solver, state)


def _last_block_point(shape, back=1):
    """(i, j, k) of a point in the kernel's last-but-(back-1) block of 3-D
    points, in the (nx, ny, nz) C order the kernel walks."""
    n3 = int(np.prod(shape))
    nblocks = -(-n3 // CHUNK)
    flat = min(n3 - 1, (nblocks - back) * CHUNK + CHUNK // 3)
    return np.unravel_index(flat, shape)


@pytest.mark.parametrize("edit", [
    lambda s: None,
    lambda s: s["S"].__setitem__(_last_block_point(s["S"].shape), np.nan),
    lambda s: s["u"].__setitem__(_last_block_point(s["u"].shape), np.nan),
    lambda s: s["u"].__setitem__(_last_block_point(s["u"].shape, 2), -13.0),
    lambda s: s["v"].__setitem__(_last_block_point(s["v"].shape), 10.25),
    lambda s: s["v"].__setitem__(_last_block_point(s["v"].shape), np.inf),
    lambda s: s["eta"].__setitem__((s["eta"].shape[0] - 1, s["eta"].shape[1] - 2), -18.0),
    lambda s: s["eta"].__setitem__((s["eta"].shape[0] - 3, s["eta"].shape[1] - 1), np.nan),
])
def test_noalloc_multi_block_matches_monitor_twice(multi, edit):
    solver, base = multi
    assert int(np.prod(base["u"].shape)) > 6 * CHUNK
    state = {k: np.array(v) for k, v in base.items()}
    edit(state)
    _check(solver, state)


def test_noalloc_checks_ice(multi):
    solver, base = multi
    state = {k: np.array(v) for k, v in base.items()}
    ice = np.zeros(state["eta"].shape, np.float32)
    _check(solver, state, ice=ice)
    ice[-1, -1] = np.inf
    _check(solver, state, ice=ice)


def test_noalloc_inclusive_limits(small):
    import torch
    solver, base = small
    state = {k: np.array(v) for k, v in base.items()}
    state["u"][0, 0, 0] = 10.0
    fields = gu.to_device(state)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert _noalloc(solver.lib, fields, solver.shape, stream, inclusive=0)[1] == 0
    assert _noalloc(solver.lib, fields, solver.shape, stream, inclusive=1)[1] == 3


def test_noalloc_rejects_fields_above_the_maximum(small):
    import torch
    solver, base = small
    fields = gu.to_device(base)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc, _, _ = _noalloc(solver.lib, fields, (4096, 4096, 16), stream)
    assert rc == _native.ZM_ERR_INVALID
