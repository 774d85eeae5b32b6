"""Load the golden fixtures of ``tests/golden`` into grid objects."""
from __future__ import annotations

import ast
import os

import numpy as np

from zhenmode_b200.config import GlobalOceanGrid, PhysicsConfig

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def grid_from(data):
    wm3 = data["grid_wet_mask_3d"]
    nx, ny, nz = wm3.shape
    z = data["grid_z"]
    wm = data["grid_wet_mask"]
    return GlobalOceanGrid(lon=data["grid_lon"], lat=data["grid_lat"], dx_2d=data["grid_dx_2d"],
                           dy=float(data["grid_dy"]), cos_lat=data["grid_cos_lat"], f=data["grid_f"],
                           z=z, dz=np.abs(np.diff(z)), nz=nz, depth=data["grid_depth"], wet_mask=wm,
                           ocean_mask=wm > 0.5, land_mask=wm < 0.5, wet_mask_3d=wm3, nx=nx, ny=ny)


def case_inputs(data):
    """(grid, physics, dt, options, state) of a step fixture."""
    grid = grid_from(data)
    physics = PhysicsConfig(**ast.literal_eval(str(data["physics"])))
    options = ast.literal_eval(str(data["options"]))
    lat = np.radians(np.asarray(grid.lat))
    tau_x = np.broadcast_to((0.1 * np.sin(2 * lat) * np.cos(lat))[None, :], (grid.nx, grid.ny)).copy()
    zeros = np.zeros((grid.nx, grid.ny))
    q_heat = np.array(data["forcing_q"]) if "forcing_q" in data else zeros.copy()
    options.update(forcing=(tau_x, zeros, q_heat), dt_bt=float(data["dt_bt"]))
    restore = float(data["restore_days"])
    if restore > 0:
        options.update(coastal_restore_mask=np.asarray(grid.wet_mask), coastal_restore_days=restore,
                       coastal_restore_T=np.array(data["in_T"][:, :, 0]))
    if "clim_T" in data:  # the sponge's relaxation targets (factory.py:470-483)
        options.update(T_init=data["clim_T"], S_init=data["clim_S"])
    for key in data:  # array-valued options of the fixture (forcing targets, masks)
        if key.startswith("arr_"):
            options[key[4:]] = data[key]
    state = {k: data["in_" + k] for k in ("u", "v", "T", "S", "eta")}
    return grid, physics, float(data["dt"]), options, state


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / den) if den > 0 else float(np.linalg.norm(a - b))
