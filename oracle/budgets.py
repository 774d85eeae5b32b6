"""ORACLE (test infrastructure only): float64 restatement of the reference's
run-level budget snapshot, ``compute_budget_diagnostics``
(src/zhenmode/model/diagnostics/snapshot.py:67-128) with the legacy
``node_thickness`` (snapshot.py:42-64) and the linear thermodynamics.

Only ``tests/`` import this module.  Parity status: pinned against the
reference's own values in ``tests/golden/diagnostics_48x24x10.npz``.
"""
from __future__ import annotations

import numpy as np

from .params import C_P, RHO_0

FIELDS = ("mean_T", "mean_S", "mean_T_top", "mean_S_top", "heat_content_J", "salt_content_kg",
          "total_volume_m3", "mean_depth_m")


def node_thickness(z):
    """snapshot.py:42-64, legacy: end nodes take the adjacent interval, interior
    nodes the mean of the two adjacent intervals."""
    dz = np.abs(np.diff(np.asarray(z, dtype=np.float64)))
    return np.concatenate(([dz[0]], 0.5 * (dz[:-1] + dz[1:]), [dz[-1]]))


def budget_diagnostics(T, S, dx_2d, dy, z, wet_mask, wet_mask_3d, rho0=RHO_0, cp=C_P):
    """snapshot.py:67-128 for the legacy geometry; returns a dict keyed like
    ``BudgetDiagnostics.as_dict``."""
    T = np.asarray(T, dtype=np.float64)
    S = np.asarray(S, dtype=np.float64)
    area = np.asarray(dx_2d, dtype=np.float64) * float(dy)
    wet3 = np.asarray(wet_mask_3d, dtype=np.float64)
    volume = (area[:, :, None] * node_thickness(z)[None, None, :]) * wet3
    total_volume = float(volume.sum())
    surface_area = area * np.asarray(wet_mask, dtype=np.float64)
    surface_total = float(surface_area.sum())
    return {
        "mean_T": float((T * volume).sum() / total_volume),
        "mean_S": float((S * volume).sum() / total_volume),
        "mean_T_top": float((T[:, :, 0] * surface_area).sum() / surface_total),
        "mean_S_top": float((S[:, :, 0] * surface_area).sum() / surface_total),
        "heat_content_J": float((rho0 * cp * T * volume).sum()),
        "salt_content_kg": float((rho0 * (S / 1000.0) * volume).sum()),
        "total_volume_m3": total_volume,
        "mean_depth_m": total_volume / float(area.sum()),
    }
