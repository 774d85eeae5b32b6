"""FP64 stage/source ledger of the B200 step: the budget audit mode of the
reference (src/zhenmode/model/diagnostics/budgets.py).

``make_budget_step(params)`` (budgets.py:264-288) takes the ``params`` that
``make_solver_global(..., return_params=True)`` returns (a ``B200Params``
carrying its step; the reference runtime passes it at runtime/run.py:113 when
``RunServices.make_budget_step`` is this function) or the ``step`` callable
itself and gives ``advance(state, forcing=None, atmosphere=None,
surface_pressure_pa=None) -> (new state, ledger)``.  The step is the ordinary
B200 step run once without the CUDA graph, with compensated float64
reductions at the reference's hook points (``zm_ledger_step``); the ledger
has the reference's keys, shapes and residual identities (budgets.py:214-262):
per-stage heat / salt / volume changes, source inputs, nonlinear process
changes, the surface advective flux, the column-projection norms and the
derived residuals.  The audits that only the non-legacy column geometries
fill (transport consistency, bottom-drag half steps) are zero, as in the
reference's legacy path.  ``forcing`` replaces (tau_x, tau_y, Q_heat) for
that call only; a runtime ``atmosphere`` or surface load is not implemented.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native

METRIC_NAMES = ("fixed_node_water_ice_enthalpy_J", "water_salt_kg", "eta_volume_m3")
STAGE_NAMES = ("linear_diffusion", "sponge", "nonlinear", "free_surface", "polar_cap_and_masks", "dynamic_ice")
SOURCE_NAMES = ("prescribed_heat", "bulk_heat", "coastal_bulk_heat", "temperature_restore", "salinity_restore",
                "prescribed_brine", "sponge", "ice_atmosphere_heat", "ice_brine")
NONLINEAR_PROCESS_NAMES = ("advection", "convection", "gm", "redi")
TRANSPORT_METRIC_NAMES = ("local_continuity_residual_m", "nontransport_eta_change_m",
                          "tracer_face_mean_mismatch_m2_per_s", "final_filter_face_change_m2_per_s")
MAXIMUM_BUDGET_FIELDS = ("projection_relative_residual_max", "transport_consistency_max",
                         "bottom_drag_face_change_max_m2_per_s")
LEDGER_COUNT = 75


def empty_budget():
    """Zero totals for interval accumulation (budgets.py:34-57)."""
    z3 = lambda: np.zeros(3)  # noqa: E731
    return {"observed_change": z3(), "stage_changes": np.zeros((len(STAGE_NAMES), 3)),
            "source_inputs": np.zeros((len(SOURCE_NAMES), 3)), "decomposition_residual": z3(),
            "budget_residual": z3(), "absolute_decomposition_residual": z3(), "absolute_budget_residual": z3(),
            "change_scale": z3(), "nonlinear_process_changes": np.zeros((len(NONLINEAR_PROCESS_NAMES), 3)),
            "nonlinear_process_scale": z3(), "advection_boundary_changes": z3(),
            "advection_boundary_residual": z3(), "absolute_advection_boundary_residual": z3(),
            "nonlinear_accounting_residual": z3(), "absolute_nonlinear_accounting_residual": z3(),
            "surface_displacement_tracer_change": z3(), "projection_transport_norm_squared": np.zeros(2),
            "projection_relative_residual_max": np.float64(0.0), "transport_consistency_max": np.zeros(4),
            "transport_audited_steps": np.float64(0.0), "bottom_drag_reference_energy_loss_J": np.float64(0.0),
            "bottom_drag_face_change_max_m2_per_s": np.float64(0.0), "bottom_drag_audited_halves": np.float64(0.0)}


def accumulate_budget(totals, interval):
    """Sum intervals, keeping the worst residual ratios (budgets.py:59-60)."""
    return {k: (np.maximum(totals[k], interval[k]) if k in MAXIMUM_BUDGET_FIELDS else totals[k] + interval[k])
            for k in totals}


def ledger_from_raw(raw):
    """The reference's ledger dict (budgets.py:234-262) from the raw sums of
    ``zm_ledger_step`` (layout in include/zm_b200.h)."""
    raw = np.asarray(raw, dtype=np.float64)
    stages = raw[0:18].reshape(6, 3)
    sources = raw[21:48].reshape(9, 3)
    processes = raw[48:60].reshape(4, 3)
    advb = raw[63:66]
    observed = raw[69:72]
    decomposition = observed - np.sum(stages, axis=0)
    budget = observed - np.sum(sources, axis=0)
    boundary = processes[0] - advb
    nonlinear = stages[2] - np.sum(sources[:6], axis=0) - np.sum(processes, axis=0)
    out = empty_budget()
    out.update({"observed_change": observed, "stage_changes": stages, "source_inputs": sources,
                "decomposition_residual": decomposition, "budget_residual": budget,
                "absolute_decomposition_residual": np.abs(decomposition), "absolute_budget_residual": np.abs(budget),
                "change_scale": raw[18:21].copy(), "nonlinear_process_changes": processes,
                "nonlinear_process_scale": raw[60:63].copy(), "advection_boundary_changes": advb.copy(),
                "advection_boundary_residual": boundary, "absolute_advection_boundary_residual": np.abs(boundary),
                "nonlinear_accounting_residual": nonlinear,
                "absolute_nonlinear_accounting_residual": np.abs(nonlinear),
                "surface_displacement_tracer_change": raw[72:75].copy(),
                "projection_transport_norm_squared": raw[66:68].copy(),
                "projection_relative_residual_max": np.float64(raw[68])})
    return out


def make_budget_step(params):
    """(state, forcing=None, atmosphere=None, surface_pressure_pa=None) ->
    (new state, ledger) for the B200 step (budgets.py:264-288)."""
    import torch

    from .solver import JaxStateG, UnsupportedOption, _torch_state_ptrs

    if isinstance(params, dict):
        step = params["step"]
    else:
        step = getattr(params, "step", params)  # the params of make_solver_global, or the step itself
    solver = step.solver
    changed = [False]

    def advance(state, forcing=None, atmosphere=None, surface_pressure_pa=None):
        if atmosphere is not None or surface_pressure_pa is not None:
            raise UnsupportedOption("runtime T_atm / surface pressure are not implemented on the B200 path")
        if forcing is not None:
            if len(forcing) != 3:
                raise ValueError("forcing must contain tau_x, tau_y and Q_heat")
            step.set_forcing(*forcing)
            changed[0] = True
        elif changed[0]:
            zeros = np.zeros(solver.shape[:2])
            step.set_forcing(*[zeros if a is None else a for a in step.factory_forcing])
            changed[0] = False
        host = isinstance(state.u, np.ndarray)
        if host:
            dev = JaxStateG(*[torch.as_tensor(np.ascontiguousarray(getattr(state, k), dtype=np.float32),
                                              device="cuda") for k in ("u", "v", "T", "S", "eta")], state.ice)
        else:
            dev = state
        fin = _torch_state_ptrs(dev, solver.shape)
        out = [torch.empty_like(t) for t in fin]
        raw = (ctypes.c_double * LEDGER_COUNT)()
        sin = _native.ZmState(*[t.data_ptr() for t in fin])
        sout = _native.ZmState(*[t.data_ptr() for t in out])
        stream = ctypes.c_void_p(torch.cuda.current_stream(fin[0].device).cuda_stream)
        solver.check(solver.lib.zm_ledger_step(solver.handle, stream, ctypes.byref(sin), ctypes.byref(sout), raw,
                                               LEDGER_COUNT), "zm_ledger_step")
        if host:
            out = [t.cpu().numpy() for t in out]
        return JaxStateG(*out, state.ice), ledger_from_raw(np.frombuffer(raw, dtype=np.float64))

    return advance
