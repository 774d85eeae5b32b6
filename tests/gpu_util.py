"""Helpers for the GPU parity tests: run the CUDA step through the C ABI on
torch device buffers and compare with the float64 oracle."""
from __future__ import annotations

import ctypes

import numpy as np

from oracle import params as oparams
from oracle import step as ostep
from zhenmode_b200 import _native, make_solver_global

FIELDS = ("u", "v", "T", "S", "eta")


def build_pair(grid, physics, dt, options):
    """(gpu step, oracle params) for one configuration."""
    opts = dict(options)
    opts["dtype"] = "float32"
    gpu = make_solver_global(grid, physics, dt, **opts)[0]
    oopts = {k: v for k, v in options.items() if k in oparams.SUPPORTED}
    oopts["dtype"] = "float64"
    return gpu, oparams.build_params(grid, physics, dt, **oopts)


def f32(state):
    """The state rounded to float32 values (the GPU's input bits), as float64."""
    return {k: np.asarray(state[k], dtype=np.float32).astype(np.float64) for k in FIELDS}


def to_device(state):
    import torch
    return [torch.as_tensor(np.ascontiguousarray(state[k], dtype=np.float32), device="cuda") for k in FIELDS]


def run_stage(gpu_step, stage, state):
    """Stage 1 = L(dt/2), 2 = N(dt), 3 = full step, via zm_run_stage."""
    import torch
    solver = gpu_step.solver
    fin = to_device(state)
    out = [torch.empty_like(t) for t in fin]
    sin = _native.ZmState(*[t.data_ptr() for t in fin])
    sout = _native.ZmState(*[t.data_ptr() for t in out])
    stream = torch.cuda.current_stream().cuda_stream
    solver.check(solver.lib.zm_run_stage(solver.handle, ctypes.c_void_p(stream), stage, ctypes.byref(sin),
                                         ctypes.byref(sout)), "zm_run_stage")
    torch.cuda.synchronize()
    return {k: t.double().cpu().numpy() for k, t in zip(FIELDS, out)}


def run_steps(gpu_step, state, nsteps):
    """nsteps full steps through zm_step (device pointers)."""
    import torch
    from zhenmode_b200 import JaxStateG
    st = JaxStateG(*to_device(state), 0.0)
    out = gpu_step.advance(st, nsteps)
    torch.cuda.synchronize()
    return {k: getattr(out, k).double().cpu().numpy() for k in FIELDS}


def rel_l2(a, b, mask=None):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if mask is not None:
        a = a * mask
        b = b * mask
    den = np.linalg.norm(b)
    num = np.linalg.norm(a - b)
    return float(num / den) if den > 0 else float(num)


def errors(got, want, fields=FIELDS):
    return {k: rel_l2(got[k], want[k]) for k in fields}
