"""FP64 stage/source ledger of one step, restated over the oracle step.

Test infrastructure (the checker of the GPU ledger), not product code.

Follows the reference's budget audit (src/zhenmode/model/diagnostics/budgets.py):
``_StageRecorder`` (:62-232) records, during one step, the heat / salt /
volume change of every accepted stage, the surface and sponge sources, the
nonlinear process tendencies (advection, convection, GM, Redi), the
advective flux through the surface and the column-projection norms;
``result`` (:234-262) forms the residual identities, ``make_budget_step``
(:264-288) returns (new state, ledger), ``empty_budget`` / ``accumulate_budget``
(:34-60) sum intervals.  The hooks fire at the places of the legacy
mode-split step: timestepping/step.py:138-161 (linear half step),
dynamics/tendencies.py:211-214 (each tracer residual), step.py:298-300 (the
projection), step.py:366-368, 425-427, 452-455 (nonlinear, free surface,
polar cap and masks, dynamic ice).
"""
from __future__ import annotations

import numpy as np

from .params import C_P, RHO_0

METRIC_NAMES = ("fixed_node_water_ice_enthalpy_J", "water_salt_kg", "eta_volume_m3")
STAGE_NAMES = ("linear_diffusion", "sponge", "nonlinear", "free_surface", "polar_cap_and_masks", "dynamic_ice")
SOURCE_NAMES = ("prescribed_heat", "bulk_heat", "coastal_bulk_heat", "temperature_restore", "salinity_restore",
                "prescribed_brine", "sponge", "ice_atmosphere_heat", "ice_brine")
NONLINEAR_PROCESS_NAMES = ("advection", "convection", "gm", "redi")
MAXIMUM_BUDGET_FIELDS = ("projection_relative_residual_max", "transport_consistency_max",
                         "bottom_drag_face_change_max_m2_per_s")
RHO_ICE, LATENT = 917.0, 3.34e5


def empty_ledger():
    """budgets.py:34-57: zero totals for interval accumulation."""
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


def accumulate(totals, interval):
    """budgets.py:59-60: sums, except the running maxima of the worst ratios."""
    return {k: (np.maximum(totals[k], interval[k]) if k in MAXIMUM_BUDGET_FIELDS else totals[k] + interval[k])
            for k in totals}


class Recorder:
    """budgets.py:62-232 for the legacy mode-split step (no ice, no GM/Redi,
    no bottom-drag half steps, no transport audit)."""

    def __init__(self, p):
        self.p = p
        self.cp = C_P
        area = np.asarray(p.dx_2d, dtype=np.float64) * float(p.dy)
        self.surface_area = area * p.wet_mask
        self.volume = area[:, :, None] * np.asarray(p.dz_node) * p.wet_mask_z
        self.stages = {n: np.zeros(3) for n in STAGE_NAMES}
        self.sources = {n: np.zeros(3) for n in SOURCE_NAMES}
        self.change_scale = np.zeros(3)
        self.processes = {n: np.zeros(3) for n in NONLINEAR_PROCESS_NAMES}
        self.process_scale = np.zeros(3)
        self.advection_boundary = np.zeros(3)
        self.projection_norm_squared = np.zeros(2)
        self.projection_relative_residual_max = 0.0

    def difference(self, before, after):
        """budgets.py:122-136: (enthalpy - latent, salt, displacement) and the
        sums of magnitudes."""
        heat = RHO_0 * self.cp * (after["T"] - before["T"]) * self.volume
        ice_b, ice_a = before.get("ice", 0.0), after.get("ice", 0.0)
        latent = RHO_ICE * LATENT * (np.asarray(ice_a) - np.asarray(ice_b)) * self.surface_area
        salt = RHO_0 / 1000.0 * (after["S"] - before["S"]) * self.volume
        disp = (after["eta"] - before["eta"]) * self.surface_area
        change = np.array([np.sum(heat) - np.sum(latent), np.sum(salt), np.sum(disp)])
        scale = np.array([np.sum(np.abs(heat)) + np.sum(np.abs(latent)), np.sum(np.abs(salt)),
                          np.sum(np.abs(disp))])
        return change, scale

    def stage(self, name, before, after):
        change, scale = self.difference(before, after)
        self.stages[name] = self.stages[name] + change
        self.change_scale = self.change_scale + scale

    def surface_sources(self, tendencies):
        """budgets.py:143-149 over dt/2 (each of the two RK2 residuals)."""
        interval = self.p.dt / 2.0
        for index, tendency in enumerate(tendencies):
            factor = RHO_0 * self.cp if index < 4 else RHO_0 / 1000.0
            amount = np.sum(tendency * self.volume) * factor * interval
            self.sources[SOURCE_NAMES[index]][0 if index < 4 else 1] += amount

    def nonlinear_terms(self, tendencies):
        """budgets.py:151-167 over dt/2."""
        interval = self.p.dt / 2.0
        for name, (ct, cs) in zip(NONLINEAR_PROCESS_NAMES, tendencies):
            heat = RHO_0 * self.cp * interval * ct * self.volume
            salt = RHO_0 / 1000.0 * interval * cs * self.volume
            self.processes[name] = self.processes[name] + np.array([np.sum(heat), np.sum(salt), 0.0])
            self.process_scale = self.process_scale + np.array([np.sum(np.abs(heat)), np.sum(np.abs(salt)), 0.0])

    def advection_boundary_fluxes(self, top_T, top_S):
        """budgets.py:169-173 over dt/2."""
        interval = self.p.dt / 2.0
        heat = RHO_0 * self.cp * interval * np.sum(top_T * self.surface_area)
        salt = RHO_0 / 1000.0 * interval * np.sum(top_S * self.surface_area)
        self.advection_boundary = self.advection_boundary + np.array([heat, salt, 0.0])

    def column_projection(self, before_top, after_top):
        """budgets.py:175-183 from the surface transports before and after."""
        norms = np.array([np.sum(before_top ** 2 * self.surface_area), np.sum(after_top ** 2 * self.surface_area)])
        self.projection_norm_squared = self.projection_norm_squared + norms
        if norms[0] > 0.0:
            rel = float(np.sqrt(norms[1] / norms[0]))
        else:
            rel = 0.0 if norms[1] == 0.0 else np.inf
        self.projection_relative_residual_max = max(self.projection_relative_residual_max, rel)

    def surface_displacement_change(self, before, after):
        """budgets.py:185-194."""
        t = after["eta"] * after["T"][..., 0] - before["eta"] * before["T"][..., 0]
        s = after["eta"] * after["S"][..., 0] - before["eta"] * before["S"][..., 0]
        return np.array([RHO_0 * self.cp * np.sum(t * self.surface_area),
                         RHO_0 / 1000.0 * np.sum(s * self.surface_area), 0.0])

    def sponge_sources(self, before, decay):
        """budgets.py:196-204."""
        fraction = 1.0 - decay
        t = (self.p.T_clim_3d - before["T"]) * fraction
        s = (self.p.S_clim_3d - before["S"]) * fraction
        self.sources["sponge"] = self.sources["sponge"] + np.array(
            [RHO_0 * self.cp * np.sum(t * self.volume), RHO_0 / 1000.0 * np.sum(s * self.volume), 0.0])

    def result(self, before, after):
        """budgets.py:214-262."""
        observed, _ = self.difference(before, after)
        stages = np.stack([self.stages[n] for n in STAGE_NAMES])
        sources = np.stack([self.sources[n] for n in SOURCE_NAMES])
        decomposition = observed - np.sum(stages, axis=0)
        budget = observed - np.sum(sources, axis=0)
        processes = np.stack([self.processes[n] for n in NONLINEAR_PROCESS_NAMES])
        boundary = self.processes["advection"] - self.advection_boundary
        nonlinear = self.stages["nonlinear"] - np.sum(sources[:6], axis=0) - np.sum(processes, axis=0)
        out = empty_ledger()
        out.update({"observed_change": observed, "stage_changes": stages, "source_inputs": sources,
                    "decomposition_residual": decomposition, "budget_residual": budget,
                    "absolute_decomposition_residual": np.abs(decomposition),
                    "absolute_budget_residual": np.abs(budget), "change_scale": self.change_scale,
                    "nonlinear_process_changes": processes, "nonlinear_process_scale": self.process_scale,
                    "advection_boundary_changes": self.advection_boundary,
                    "advection_boundary_residual": boundary,
                    "absolute_advection_boundary_residual": np.abs(boundary),
                    "nonlinear_accounting_residual": nonlinear,
                    "absolute_nonlinear_accounting_residual": np.abs(nonlinear),
                    "surface_displacement_tracer_change": self.surface_displacement_change(before, after),
                    "projection_transport_norm_squared": self.projection_norm_squared,
                    "projection_relative_residual_max": np.float64(self.projection_relative_residual_max)})
        return out


def ledger_step(st, p):
    """budgets.py:264-288 ``make_budget_step``'s advance: (new state, ledger)."""
    from . import step as ostep
    rec = Recorder(p)
    new = ostep.step(st, p, rec=rec)
    return new, rec.result(st, new)
