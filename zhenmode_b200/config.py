"""Physical constants and the grid / physics configuration objects.

These mirror ZhenMode's own configuration types field for field so that a
caller can hand either this module's objects or the reference's objects to
:func:`zhenmode_b200.make_solver_global` (duck typing on attribute names):

* constants: ``src/zhenmode/model/config.py:12-25``
* ``GlobalOceanGrid``: ``src/zhenmode/model/solver/geometry/grid.py:13-61``
* ``PhysicsConfig``: ``src/zhenmode/model/config.py:86-140``
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

G_EARTH = 9.81          # m/s^2
RHO_0 = 1025.0          # kg/m^3 reference seawater density
ALPHA_T = 2.0e-4        # 1/degC thermal expansion
BETA_S = 7.6e-4         # 1/psu haline contraction
C_P = 3992.0            # J/(kg degC)
R_EARTH = 6371.0e3      # m
OMEGA = 7.2921e-5       # rad/s


@dataclass
class GlobalOceanGrid:
    """Global lon-lat grid; 2-D arrays are ``(nx, ny)``, 3-D ``(nx, ny, nz)``.

    Longitude (axis 0) is periodic, latitude (axis 1) is closed; ``z`` is
    negative downward with ``z[0]`` the surface node.
    """
    lon: np.ndarray
    lat: np.ndarray
    dx_2d: np.ndarray
    dy: float
    cos_lat: np.ndarray
    f: np.ndarray
    z: np.ndarray
    dz: np.ndarray
    nz: int
    depth: np.ndarray
    wet_mask: np.ndarray
    ocean_mask: np.ndarray
    land_mask: np.ndarray
    wet_mask_3d: np.ndarray
    nx: int
    ny: int


@dataclass(frozen=True)
class PhysicsConfig:
    """Hydrostatic primitive-equation physics coefficients (SI units)."""
    nu_h: float = 100.0
    nu_v: float = 1.0e-4
    kappa_h: float = 100.0
    kappa_v: float = 1.0e-5
    kappa_conv: float = 0.05
    nu_bi: float = 1.0e12
    kappa_bi: float = 1.0e12
    kappa_gm: float = 0.0
    gm_slope_max: float = 0.01
    kappa_redi: float = 0.0
    T_ref: float = 15.0
    S_ref: float = 35.0
    tau_x: float = 0.0
    tau_y: float = 0.0
    Q_heat: float = 0.0
    cd: float = 2.5e-3
    r_bot: float = 1.0e-3
    bottom_friction: str = 'linear'
    thermodynamics: str = 'linear'
