"""Seeded synthetic inputs for the global ocean step (grid, bathymetry, T/S,
wind stress) at any resolution.

The reference runs on ETOPO/WOA/NCEP data that is not shipped; every workload
here is synthetic, built by coordinates (not by index) so one generator gives
consistent fields at 4 deg, 2 deg, 1 deg, 0.5 deg and 0.45 deg:

* grid metrics follow the area layout of ``build_global_grid``
  (``src/zhenmode/model/solver/geometry/grid.py:291-380``): cell-centred
  longitudes ``(i+1/2) 360/nx``, latitudes ``-90+(j+1/2) 180/ny``,
  ``dx = R cos(lat) dlon``, ``dy = R dlat``, ``f = 2 Omega sin(lat)``, a 3-D wet
  mask ``|z_k| <= depth`` and the default minimum depth ``|z[1]|``;
* bathymetry is 3000 m plus twelve seeded Gaussian ridges/basins, clipped to
  5000 m, with land poleward of 65 deg (keeps the explicit CFL limits of the
  0.5 deg preset satisfiable);
* levels are stretched, 10 m at the surface, summing to 5000 m;
* T is an exponential thermocline (28 -> 2 degC, e-folding 500 m) with a
  cos(lat) surface modulation plus optional smoothed mesoscale noise; S is
  35 psu with clipped seeded noise;
* wind stress ``tau_x = 0.1 sin(2 lat) cos(lat)`` N/m^2.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from .config import OMEGA, R_EARTH, GlobalOceanGrid, PhysicsConfig


def stretched_levels(nz, total_depth=5000.0, dz_top=10.0, power=1.6245):
    """Level depths z (nz,), z[0]=0, thicknesses dz_top + A (k/(nz-2))^power.

    A is solved so the thicknesses sum to ``total_depth``; at nz=50 this is the
    10 m -> 250 m profile (A = 240).
    """
    if nz < 3:
        raise ValueError("need at least three levels")
    k = np.arange(nz - 1, dtype=np.float64)
    shape = (k / (nz - 2)) ** power
    amplitude = (total_depth - dz_top * (nz - 1)) / shape.sum()
    dz = dz_top + amplitude * shape
    z = -np.concatenate(([0.0], np.cumsum(dz)))
    z[-1] = -total_depth
    return z


def _great_circle_deg(lon, lat, lon_c, lat_c):
    la, lb = np.radians(lat), np.radians(lat_c)
    dl = np.radians(lon - lon_c)
    cosd = np.sin(la) * np.sin(lb) + np.cos(la) * np.cos(lb) * np.cos(dl)
    return np.degrees(np.arccos(np.clip(cosd, -1.0, 1.0)))


def synthetic_bathymetry(lon, lat, seed=1, features=12, land_lat=65.0,
                         base=3000.0, max_depth=5000.0):
    """Depth (nx, ny) in metres; <= 0 marks land."""
    rng = np.random.default_rng(seed)
    amp = rng.uniform(-2500.0, 2500.0, features)
    sigma = rng.uniform(5.0, 25.0, features)
    lon_c = rng.uniform(0.0, 360.0, features)
    lat_c = np.degrees(np.arcsin(rng.uniform(-1.0, 1.0, features)))
    lon2, lat2 = np.meshgrid(lon, lat, indexing='ij')
    depth = np.full(lon2.shape, base)
    for a, s, lc, pc in zip(amp, sigma, lon_c, lat_c):
        d = _great_circle_deg(lon2, lat2, lc, pc)
        depth += a * np.exp(-d * d / (2.0 * s * s))
    depth = np.minimum(depth, max_depth)
    depth[np.abs(lat2) > land_lat] = 0.0
    return depth


def build_grid(nx, ny, nz, seed=1, land_lat=65.0, z=None, depth=None):
    """A GlobalOceanGrid with seeded synthetic bathymetry."""
    lon = (np.arange(nx) + 0.5) * 360.0 / nx
    lat = -90.0 + (np.arange(ny) + 0.5) * 180.0 / ny
    if z is None:
        z = stretched_levels(nz)
    z = np.asarray(z, dtype=np.float64)
    if depth is None:
        depth = synthetic_bathymetry(lon, lat, seed=seed, land_lat=land_lat)
    min_depth = float(abs(z[1]))
    depth = np.where(depth > 0.0, np.where(depth < min_depth, 0.0, depth), 0.0)
    cos_lat = np.cos(np.radians(lat))
    dx_2d = np.broadcast_to(R_EARTH * np.radians(360.0 / nx) * cos_lat, (nx, ny)).copy()
    dy = float(R_EARTH * np.radians(180.0 / ny))
    f = np.broadcast_to(2.0 * OMEGA * np.sin(np.radians(lat))[None, :], (nx, ny)).copy()
    ocean = depth > 0.0
    wet3 = ((np.abs(z)[None, None, :] <= depth[:, :, None]) & ocean[:, :, None]).astype(np.float64)
    return GlobalOceanGrid(lon=lon, lat=lat, dx_2d=dx_2d, dy=dy, cos_lat=cos_lat, f=f,
                           z=z, dz=np.abs(np.diff(z)), nz=int(nz), depth=depth,
                           wet_mask=ocean.astype(np.float64), ocean_mask=ocean,
                           land_mask=~ocean, wet_mask_3d=wet3, nx=int(nx), ny=int(ny))


def _binomial_smooth(field, passes):
    """[1,2,1]/4 passes, periodic in x (axis 0), edge-held in y (axis 1)."""
    out = np.array(field, dtype=np.float64)
    for _ in range(passes):
        out = 0.25 * (np.roll(out, 1, 0) + 2.0 * out + np.roll(out, -1, 0))
        pad = np.concatenate((out[:, :1], out, out[:, -1:]), axis=1)
        out = 0.25 * (pad[:, :-2] + 2.0 * pad[:, 1:-1] + pad[:, 2:])
    return out


def initial_fields(grid, perturb_sigma=0.0, seed_T=2, seed_S=3, smooth_deg=1.0):
    """Initial (T, S), shape (nx, ny, nz), float64."""
    nx, ny, nz = grid.nx, grid.ny, grid.nz
    z = np.asarray(grid.z)
    cos_lat = np.asarray(grid.cos_lat)
    profile = np.exp(z / 500.0)
    T = 2.0 + 26.0 * cos_lat[None, :, None] * profile[None, None, :] * np.ones((nx, 1, 1))
    if perturb_sigma > 0.0:
        rng = np.random.default_rng(seed_T)
        noise = rng.standard_normal((nx, ny))
        cells = smooth_deg / (180.0 / ny)
        noise = _binomial_smooth(noise, int(round(2.0 * cells * cells)))
        wet = np.asarray(grid.wet_mask) > 0.5
        std = float(np.std(noise[wet])) if np.any(wet) else 1.0
        noise = noise / max(std, 1e-30)
        T = T + perturb_sigma * noise[:, :, None] * profile[None, None, :]
    rng = np.random.default_rng(seed_S)
    S = 35.0 + np.clip(0.1 * rng.standard_normal((nx, ny, nz)), -0.5, 0.5)
    return T, S


def wind_forcing(grid, amplitude=0.1):
    """(tau_x, tau_y, Q_heat) each (nx, ny)."""
    lat = np.radians(np.asarray(grid.lat))
    tau_x = amplitude * np.sin(2.0 * lat) * np.cos(lat)
    tau_x = np.broadcast_to(tau_x[None, :], (grid.nx, grid.ny)).copy()
    zeros = np.zeros((grid.nx, grid.ny))
    return tau_x, zeros, zeros.copy()


# Option sets.  ``plain`` is the 0.5 deg restoring production preset
# (configs/zhenmode/presets/global-050deg-restoring.yaml:10-38 with the
# resolution auto-scaling of src/zhenmode/model/runtime/cli.py:48-60), without
# the column projection.  ``smoke`` is configs/zhenmode/presets/synthetic-smoke.yaml.
PLAIN_PHYSICS = PhysicsConfig(nu_h=2.0e6, nu_v=1.0e-4, kappa_h=100.0, kappa_v=1.0e-6,
                              kappa_conv=0.01, nu_bi=1.25e13, kappa_bi=1.25e13,
                              kappa_gm=0.0, kappa_redi=0.0, r_bot=1.0e-3)
PLAIN_OPTIONS = dict(mode_split=True, use_scan=True, localize_conv=True, fct_adv=True,
                     polar_cap_rows=2, polar_cap_taper=3, lambda_bulk=0.0)
SMOKE_PHYSICS = PhysicsConfig(nu_h=0.0, nu_bi=0.0, kappa_v=0.0, kappa_conv=0.0)
SMOKE_OPTIONS = dict(mode_split=True, use_scan=True, polar_cap_rows=0, polar_cap_taper=0)


@dataclasses.dataclass
class Workload:
    name: str
    nx: int
    ny: int
    nz: int
    dt: float
    dt_bt: float
    steps: int
    physics: PhysicsConfig
    options: dict
    perturb_sigma: float
    restore_days: float
    dtype: str


WORKLOADS = {
    "smoke": Workload("smoke", 90, 45, 15, 10.0, 5.0, 8, SMOKE_PHYSICS, SMOKE_OPTIONS,
                      0.0, 0.0, "float64"),
    "plain": Workload("plain", 720, 360, 50, 1800.0, 75.0, 48, PLAIN_PHYSICS, PLAIN_OPTIONS,
                      0.2, 30.0, "float32"),
    "precision": Workload("precision", 800, 400, 50, 1800.0, 1800.0 / 27, 480,
                          dataclasses.replace(PLAIN_PHYSICS, nu_h=2.0e6 * 0.81, nu_bi=1.25e13 * 0.6561,
                                              kappa_bi=1.25e13 * 0.6561),
                          PLAIN_OPTIONS, 0.2, 30.0, "float32"),
}


def make_case(name_or_workload, nx=None, ny=None, nz=None, dtype=None):
    """Return (grid, physics, dt, kwargs, T_init, S_init) for a workload.

    ``nx/ny/nz`` rescale the named option set to another grid size (used by
    the parity tests); ``kwargs`` are ``make_solver_global`` keyword options.
    """
    wl = WORKLOADS[name_or_workload] if isinstance(name_or_workload, str) else name_or_workload
    nx = wl.nx if nx is None else nx
    ny = wl.ny if ny is None else ny
    nz = wl.nz if nz is None else nz
    grid = build_grid(nx, ny, nz)
    T, S = initial_fields(grid, perturb_sigma=wl.perturb_sigma)
    forcing = wind_forcing(grid)
    kwargs = dict(wl.options)
    kwargs.update(forcing=forcing, dt_bt=wl.dt_bt, dtype=dtype or wl.dtype)
    if wl.restore_days > 0.0:
        kwargs.update(coastal_restore_mask=np.asarray(grid.wet_mask),
                      coastal_restore_days=wl.restore_days,
                      coastal_restore_T=np.array(T[:, :, 0]))
    return grid, wl.physics, wl.dt, kwargs, T, S
