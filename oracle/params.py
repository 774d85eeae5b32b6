"""ORACLE (test infrastructure only): float64 parameter assembly for the CPU
restatement of ZhenMode's production global step.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this package; the product (``zhenmode_b200``) never does.

Restates the legacy-geometry subset of the reference factory:
``make_fd_params`` (src/zhenmode/model/solver/geometry/fd_metrics.py:9-148)
and ``make_solver_global`` (src/zhenmode/model/solver/factory.py:397-695),
with the constants of src/zhenmode/model/config.py:12-25.  Parity status: pinned
against golden vectors produced by the reference's own step code (see
``tests/golden/make_golden.py``).
"""
from __future__ import annotations

import math
from types import SimpleNamespace

import numpy as np

G_EARTH = 9.81
RHO_0 = 1025.0
ALPHA_T = 2.0e-4
BETA_S = 7.6e-4
C_P = 3992.0
R_EARTH = 6371.0e3
OMEGA = 7.2921e-5

SUPPORTED = ("mode_split", "dt_bt", "nu_nsub", "dtype", "use_scan", "forcing", "T_atm",
             "lambda_bulk", "S_ref_surf", "sss_restore_days", "coastal_restore_mask",
             "coastal_restore_days", "coastal_restore_T", "coastal_bulk_mask",
             "coastal_bulk_lambda", "coastal_kappa_h_mask", "coastal_kappa_h",
             "coastal_kappa_v_mask", "coastal_kappa_v", "sponge_days", "sponge_cells",
             "T_init", "S_init", "polar_cap_rows", "polar_cap_taper", "eta_relax_days",
             "eta_relax_box", "eta_relax_buffer", "freeze_adv_vel", "conservative_kv",
             "localize_conv", "monotone_adv", "fct_adv", "ice_freeze_temp_c", "ice_salt_flux",
             "vertical_diffusion", "project_adv_vel", "projection_niter", "projection_rtol",
             "projection_preconditioner", "projection_max_refinements")


def _coastal(mask, coefficient, shape):
    """factory.py:23-27: a masked nonnegative coefficient field, else zeros."""
    if mask is not None and coefficient > 0.0:
        return np.asarray(mask, dtype=np.float64) * coefficient
    return np.zeros(shape)


def build_params(grid, physics, dt, **opts):
    """Return a namespace with the FDPhysParams fields the legacy step reads.

    ``opts`` are ``make_solver_global`` keyword options (factory.py:30-68).
    ``vertical_diffusion`` ('explicit' | 'implicit') is an extension of this
    project: 'implicit' replaces the explicit L-step vertical diffusion by one
    backward-Euler solve per column (not a reference option).
    """
    unknown = set(opts) - set(SUPPORTED)
    if unknown:
        raise ValueError(f"oracle does not implement options {sorted(unknown)}")
    if not opts.get("mode_split", False):
        raise ValueError("oracle implements the mode-split production path only")
    nx, ny, nz = int(grid.nx), int(grid.ny), int(grid.nz)
    z = np.asarray(grid.z, dtype=np.float64)
    dzv = np.asarray(grid.dz, dtype=np.float64)
    p = SimpleNamespace(nx=nx, ny=ny, nz=nz)

    # --- metrics (fd_metrics.py:34-113) ---
    p.dx_2d = np.asarray(grid.dx_2d, dtype=np.float64)
    p.dy = float(grid.dy)
    p.cos_lat = np.asarray(grid.cos_lat, dtype=np.float64)
    p.inv_dx = (1.0 / p.dx_2d)[:, :, None]
    p.inv_dy = 1.0 / p.dy
    p.inv_dx2 = (1.0 / p.dx_2d ** 2)[:, :, None]
    p.inv_dy2 = p.inv_dy ** 2
    p.f = np.asarray(grid.f, dtype=np.float64)
    p.wet_mask = np.asarray(grid.wet_mask, dtype=np.float64)
    if getattr(grid, "wet_mask_3d", None) is not None:
        p.wet_mask_z = np.asarray(grid.wet_mask_3d, dtype=np.float64)
    else:
        p.wet_mask_z = np.broadcast_to(p.wet_mask[:, :, None], (nx, ny, nz)).copy()
    interior = np.ones(ny)
    interior[0] = interior[-1] = 0.0
    p.interior_mask_z = np.broadcast_to(interior[None, :], (nx, ny))[:, :, None]
    p.z = z
    p.dz_3d = dzv.reshape(1, 1, -1)
    p.dz_iface = np.abs(np.diff(z)).reshape(1, 1, -1)
    gaps = np.abs(np.diff(z))
    p.dz_node = np.concatenate(([gaps[0]], 0.5 * (gaps[:-1] + gaps[1:]), [gaps[-1]])).reshape(1, 1, -1)
    p.dz_surface = float(abs(z[0] - z[1]))
    p.surface_mask = np.zeros(nz)
    p.surface_mask[0] = 1.0
    p.surface_mask = p.surface_mask.reshape(1, 1, -1)
    p.bottom_mask = np.zeros(nz)
    p.bottom_mask[-1] = 1.0
    p.bottom_mask = p.bottom_mask.reshape(1, 1, -1)

    # --- physics scalars (factory.py:594-695) ---
    for name in ("nu_h", "nu_v", "kappa_h", "kappa_v", "kappa_conv", "nu_bi", "kappa_bi",
                 "T_ref", "S_ref", "r_bot", "cd"):
        setattr(p, name, float(getattr(physics, name)))
    p.bottom_friction = physics.bottom_friction
    if p.bottom_friction != "linear":
        raise ValueError("oracle implements linear bottom drag only")
    if getattr(physics, "kappa_gm", 0.0) > 0 or getattr(physics, "kappa_redi", 0.0) > 0:
        raise ValueError("oracle does not implement GM/Redi")
    if getattr(physics, "thermodynamics", "linear") != "linear":
        raise ValueError("oracle implements the linear EOS only")
    p.dt = float(dt)

    forcing = opts.get("forcing")
    if forcing is None:
        p.tau_x_2d = np.zeros((nx, ny))
        p.tau_y_2d = np.zeros((nx, ny))
        p.Q_heat_2d = np.zeros((nx, ny))
    else:
        p.tau_x_2d, p.tau_y_2d, p.Q_heat_2d = (np.array(a, dtype=np.float64) for a in forcing)

    # Shallow-water depth of the legacy column: the whole vertical span (factory.py:405-406).
    p.H_sw = float(np.sum(dzv))
    p.dz_norm = dzv.reshape(1, 1, -1) / p.H_sw

    lambda_bulk = float(opts.get("lambda_bulk", 0.0))
    T_atm = opts.get("T_atm")
    if T_atm is not None and lambda_bulk > 0.0:
        p.T_atm_3d = np.asarray(T_atm, dtype=np.float64)[:, :, None]
    else:
        p.T_atm_3d = np.zeros((nx, ny, 1))
        lambda_bulk = 0.0
    p.lambda_bulk = lambda_bulk

    S_ref_surf = opts.get("S_ref_surf")
    sss_days = float(opts.get("sss_restore_days", 0.0))
    if S_ref_surf is not None and sss_days > 0.0:
        p.S_ref_2d = np.asarray(S_ref_surf, dtype=np.float64)
        p.restore_coef_S = 1.0 / (sss_days * 86400.0)
    else:
        p.S_ref_2d = np.zeros((nx, ny))
        p.restore_coef_S = 0.0

    p.coastal_kappa_v_2d = _coastal(opts.get("coastal_kappa_v_mask"), float(opts.get("coastal_kappa_v", 0.0)), (nx, ny))
    p.coastal_kappa_h_2d = _coastal(opts.get("coastal_kappa_h_mask"), float(opts.get("coastal_kappa_h", 0.0)), (nx, ny))
    p.coastal_bulk_lambda_2d = _coastal(opts.get("coastal_bulk_mask"), float(opts.get("coastal_bulk_lambda", 0.0)), (nx, ny))
    cr_mask = opts.get("coastal_restore_mask")
    cr_days = float(opts.get("coastal_restore_days", 0.0))
    cr_T = opts.get("coastal_restore_T")
    if cr_mask is not None and cr_days > 0.0 and cr_T is not None:
        p.coastal_restore_coef_2d = np.asarray(cr_mask, dtype=np.float64) / (cr_days * 86400.0)
        p.coastal_restore_T_2d = np.asarray(cr_T, dtype=np.float64)
    else:
        p.coastal_restore_coef_2d = np.zeros((nx, ny))
        p.coastal_restore_T_2d = np.zeros((nx, ny))

    # Lateral sponge (factory.py:459-491).
    sponge_days = float(opts.get("sponge_days", 0.0))
    sponge_cells = int(opts.get("sponge_cells", 0))
    if sponge_days > 0.0 and sponge_cells > 0:
        r_max = 1.0 / (sponge_days * 86400.0)
        j = np.arange(ny)
        edge = np.minimum(j, ny - 1 - j)
        taper = np.where(edge < sponge_cells, 0.5 * (1.0 + np.cos(np.pi * edge / sponge_cells)), 0.0)
        p.sponge_rate_2d = np.broadcast_to((r_max * taper)[None, :], (nx, ny)).copy()
        wm3 = p.wet_mask_z
        T_init, S_init = opts.get("T_init"), opts.get("S_init")
        if T_init is not None:
            p.T_clim_3d = np.asarray(T_init) * wm3 + (1.0 - wm3) * p.T_ref
            S_clim = np.asarray(S_init) if S_init is not None else np.full((nx, ny, nz), p.S_ref)
            p.S_clim_3d = S_clim * wm3 + (1.0 - wm3) * p.S_ref
        else:
            p.T_clim_3d = np.full((nx, ny, nz), p.T_ref)
            p.S_clim_3d = np.full((nx, ny, nz), p.S_ref)
    else:
        p.sponge_rate_2d = np.zeros((nx, ny))
        p.T_clim_3d = np.zeros((nx, ny, nz))
        p.S_clim_3d = np.zeros((nx, ny, nz))
    p.sponge_rate = p.sponge_rate_2d[:, :, None]

    # Semi-enclosed-sea eta relaxation box (factory.py:498-521).
    relax_days = float(opts.get("eta_relax_days", 0.0))
    box = opts.get("eta_relax_box")
    if relax_days > 0.0 and box is not None:
        lon0, lon1, lat0, lat1 = box
        lon2, lat2 = np.meshgrid(np.asarray(grid.lon), np.asarray(grid.lat), indexing="ij")
        core = (lon2 >= lon0) & (lon2 <= lon1) & (lat2 >= lat0) & (lat2 <= lat1)
        d_out = np.maximum(np.maximum(np.maximum(lon0 - lon2, lon2 - lon1), 0.0),
                           np.maximum(np.maximum(lat0 - lat2, lat2 - lat1), 0.0))
        buf = float(opts.get("eta_relax_buffer", 1.0))
        mask = np.where(core, 1.0, np.where(d_out < buf, 0.5 * (1.0 + np.cos(np.pi * d_out / buf)), 0.0))
        p.eta_relax_mask = mask * p.wet_mask
        p.eta_relax_rate = 1.0 / (relax_days * 86400.0)
    else:
        p.eta_relax_mask = np.zeros((nx, ny))
        p.eta_relax_rate = 0.0

    p.polar_cap_rows = int(opts.get("polar_cap_rows", 2))
    p.polar_cap_taper = int(opts.get("polar_cap_taper", 3))
    if p.polar_cap_rows > 0 and 2 * (p.polar_cap_rows + p.polar_cap_taper) > ny:
        raise ValueError("polar cap bands must not overlap")

    # 2/3-rule dealias mask along longitude (factory.py:529-533).
    keep = max(1, int((nx // 2) * 2 / 3))
    kidx = np.fft.fftfreq(nx) * nx
    p.dealias_lon_mask = (np.abs(kidx) <= keep).astype(np.float64).reshape(nx, 1, 1)

    # Mode split (factory.py:540-545) and subcycle counts (factory.py:560-567).
    dt_bt = float(opts.get("dt_bt", 150.0))
    p.n_subcyc = max(1, int(round(dt / dt_bt)))
    p.dt_bt = dt / p.n_subcyc
    nu_nsub = opts.get("nu_nsub")
    if nu_nsub == "cfl":
        inv_dx2_max = float(np.max(p.dx_2d ** -2))
        nu_nsub = max(1, int(np.ceil(p.nu_h * (dt / 2.0) * (inv_dx2_max + p.inv_dy2) / 0.25)))
    elif nu_nsub is not None:
        nu_nsub = max(1, int(nu_nsub))
    p.nu_nsub = nu_nsub
    dz_min = float(np.min(dzv))
    p.conv_nsub = max(1, int(math.ceil(p.kappa_conv * dt / (0.4 * dz_min ** 2))))
    p.adv_nsub = max(1, int(math.ceil(dt * 4.0e-3 / (0.5 * dz_min))))

    p.freeze_adv_vel = bool(opts.get("freeze_adv_vel", False))
    p.conservative_kv = bool(opts.get("conservative_kv", False))
    p.localize_conv = bool(opts.get("localize_conv", False))
    p.monotone_adv = bool(opts.get("monotone_adv", False))
    p.fct_adv = bool(opts.get("fct_adv", False))
    p.ice_freeze_temp_c = float(opts.get("ice_freeze_temp_c", -1.8))
    p.ice_salt_flux = float(opts.get("ice_salt_flux", 0.0))
    # column projection of the stage-2 advective velocity (factory.py:366-386, 650)
    p.project_adv_vel = bool(opts.get("project_adv_vel", False))
    niter = opts.get("projection_niter")
    p.projection_niter = 150 if niter is None else int(niter)
    if p.projection_niter <= 0:
        raise ValueError("projection_niter must be a positive integer")
    rtol = opts.get("projection_rtol")
    # the tolerance floors follow the dtype the step runs in (float32 / float64)
    eps = float(np.finfo(np.float32 if opts.get("dtype", "float64") == "float32" else np.float64).eps)
    p.projection_rtol = max(float(rtol or 1e-12), 32.0 * eps)
    p.projection_transport_rtol = max(1e-10, 32.0 * eps)
    p.projection_preconditioner = opts.get("projection_preconditioner", "none")
    if p.projection_preconditioner not in ("none", "jacobi"):
        raise ValueError("projection_preconditioner must be none or jacobi")
    p.projection_max_refinements = int(opts.get("projection_max_refinements", 2))
    if not 0 <= p.projection_max_refinements <= 2:
        raise ValueError("projection_max_refinements must be an integer from 0 to 2")
    p.vertical_diffusion = opts.get("vertical_diffusion", "explicit")
    if p.vertical_diffusion not in ("explicit", "implicit"):
        raise ValueError("vertical_diffusion must be 'explicit' or 'implicit'")
    return p


def init_state(p, T_init=None, S_init=None):
    """Initial state with land and below-seafloor nodes at the T_ref/S_ref
    sentinel (factory.py:766-788); returns dict u, v, T, S, eta."""
    shape = (p.nx, p.ny, p.nz)
    T = np.full(shape, p.T_ref) if T_init is None else np.array(T_init, dtype=np.float64)
    S = np.full(shape, p.S_ref) if S_init is None else np.array(S_init, dtype=np.float64)
    wm = p.wet_mask_z
    T = T * wm + (1.0 - wm) * p.T_ref
    S = S * wm + (1.0 - wm) * p.S_ref
    return dict(u=np.zeros(shape), v=np.zeros(shape), T=T, S=S, eta=np.zeros((p.nx, p.ny)))
