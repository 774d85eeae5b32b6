"""Ensembles: several steps from ``make_solver_global`` (perturbed members,
grids of any sizes) advanced together, one CUDA-graph launch per step of
every member (``zm_ensemble_*`` in ``libzm_b200.so``)."""
from __future__ import annotations

import ctypes

from . import _native
from .solver import JaxStateG


def _stream():
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


class Ensemble:
    """Members are steps returned by ``make_solver_global``; each keeps its own
    resident state, loaded with :meth:`load` and read with :meth:`store`."""

    def __init__(self, steps):
        self.steps = list(steps)
        if not self.steps:
            raise ValueError("an ensemble needs at least one member")
        self.lib = _native.load()
        handles = (ctypes.c_void_p * len(self.steps))(*[s.solver.handle.value for s in self.steps])
        h = ctypes.c_void_p()
        rc = self.lib.zm_ensemble_create(handles, len(self.steps), ctypes.byref(h))
        if rc != _native.ZM_OK:
            raise RuntimeError(f"zm_ensemble_create failed with status {rc}")
        self.handle = h
        self.kernels_per_step = 0

    def load(self, states):
        """Make each member's resident state a copy of the given (CUDA) state."""
        if len(states) != len(self.steps):
            raise ValueError("one state per member")
        for step, st in zip(self.steps, states):
            sv = step.solver
            sin = _native.ZmState(*[getattr(st, k).data_ptr() for k in ("u", "v", "T", "S", "eta")])
            sv.check(sv.lib.zm_load_state(sv.handle, _stream(), ctypes.byref(sin)), "zm_load_state")

    def advance(self, nsteps=1):
        """nsteps steps of every member, one graph launch per step; stream ordered."""
        k = ctypes.c_int32()
        rc = self.lib.zm_ensemble_advance(self.handle, _stream(), int(nsteps), ctypes.byref(k))
        if rc != _native.ZM_OK:
            raise RuntimeError(f"zm_ensemble_advance failed with status {rc}")
        self.kernels_per_step = int(k.value)

    def store(self):
        """The members' resident states as new CUDA tensors (reference layout)."""
        import torch
        out = []
        for step in self.steps:
            sv = step.solver
            nx, ny, nz = sv.shape
            f = [torch.empty((nx, ny, nz), dtype=torch.float32, device="cuda") for _ in range(4)]
            eta = torch.empty((nx, ny), dtype=torch.float32, device="cuda")
            so = _native.ZmState(*[t.data_ptr() for t in f + [eta]])
            sv.check(sv.lib.zm_store_state(sv.handle, _stream(), ctypes.byref(so)), "zm_store_state")
            out.append(JaxStateG(*f, eta, torch.zeros_like(eta)))
        return out

    def monitor_codes(self):
        """The monitor code of every member after the last advance (synchronizes)."""
        codes = []
        for step in self.steps:
            sv = step.solver
            c = ctypes.c_int32()
            sv.check(sv.lib.zm_status(sv.handle, ctypes.byref(c)), "zm_status")
            codes.append(int(c.value))
        return codes

    def __del__(self):
        h = getattr(self, "handle", None)
        if h:
            self.lib.zm_ensemble_destroy(h)
            self.handle = None
