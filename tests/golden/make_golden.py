"""Generate golden vectors by running ZhenMode's own solver code.

Run in a container that holds the ZhenMode source tree, giving the path of
its ``src`` directory (the one that holds the ``zhenmode`` package) as the
argument or in ``ZHENMODE_SRC``::

    python tests/golden/make_golden.py --src <zhenmode-checkout>/src

JAX is not installed here, so the unmodified reference modules are imported
with the NumPy-backed stand-in under ``tests/golden/_jaxshim`` on
``sys.path`` (float64, eager).  Outputs are ``tests/golden/*.npz``; the
parity tests compare the float64 oracle (``oracle/``) and, on a GPU, the
CUDA step against them.  This script is the only reader of the reference
tree; nothing at test time needs it.
"""
from __future__ import annotations

import dataclasses
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def _ref_src():
    if "--src" in sys.argv:
        return sys.argv[sys.argv.index("--src") + 1]
    if os.environ.get("ZHENMODE_SRC"):
        return os.environ["ZHENMODE_SRC"]
    raise SystemExit("make_golden.py: give the ZhenMode source tree with --src <path>/src or ZHENMODE_SRC")


REF_SRC = _ref_src()
sys.path[:0] = [os.path.join(HERE, "_jaxshim"), REF_SRC, ROOT]

import zhenmode.model.config as ref_config  # noqa: E402
from zhenmode.model.solver.dynamics import barotropic as ref_bt  # noqa: E402
from zhenmode.model.solver.dynamics import pressure as ref_pressure  # noqa: E402
from zhenmode.model.solver.dynamics import tendencies as ref_tend  # noqa: E402
from zhenmode.model.solver.dynamics import transport as ref_transport  # noqa: E402
from zhenmode.model.solver.factory import make_solver_global  # noqa: E402
from zhenmode.model.solver.numerics import horizontal as ref_h  # noqa: E402
from zhenmode.model.solver.numerics import vertical as ref_v  # noqa: E402
from zhenmode.model.solver.physics import vertical as ref_pv  # noqa: E402
from zhenmode.model.solver.state import JaxStateG  # noqa: E402
from zhenmode.model.solver.timestepping import step as ref_step  # noqa: E402

from zhenmode_b200 import workloads  # noqa: E402


def _physics(phys):
    return ref_config.PhysicsConfig(**{f.name: getattr(phys, f.name)
                                       for f in dataclasses.fields(phys)})


def _np(x):
    return np.array(np.asarray(x), dtype=np.float64)


def _f32(x):
    """Round to float32-representable values (kept as float64): the GPU step
    holds its state in float32, so the goldens start from the same bits."""
    return np.asarray(x, dtype=np.float32).astype(np.float64)


def _smooth_noise(rng, shape, passes=2):
    a = rng.standard_normal(shape)
    for _ in range(passes):
        a = 0.25 * (np.roll(a, 1, 0) + 2 * a + np.roll(a, -1, 0))
        a = 0.25 * (np.roll(a, 1, 1) + 2 * a + np.roll(a, -1, 1))
    return a / np.std(a)


def _moving_state(grid, T, S, seed, amp_u=0.05, amp_eta=0.05):
    """Seeded nonzero wet-point velocity and free surface on top of T/S."""
    rng = np.random.default_rng(seed)
    wm = np.asarray(grid.wet_mask_3d)
    nx, ny, nz = wm.shape
    u = amp_u * _smooth_noise(rng, (nx, ny, nz)) * wm
    v = amp_u * _smooth_noise(rng, (nx, ny, nz)) * wm
    v[:, 0] = 0.0
    v[:, -1] = 0.0
    eta = amp_eta * _smooth_noise(rng, (nx, ny)) * np.asarray(grid.wet_mask)
    T = T * wm + (1 - wm) * 15.0
    S = S * wm + (1 - wm) * 35.0
    return u, v, T, S, eta


def _grid_arrays(grid):
    return dict(grid_lon=np.asarray(grid.lon), grid_lat=np.asarray(grid.lat),
                grid_dx_2d=np.asarray(grid.dx_2d), grid_dy=np.float64(grid.dy),
                grid_cos_lat=np.asarray(grid.cos_lat), grid_f=np.asarray(grid.f),
                grid_z=np.asarray(grid.z), grid_depth=np.asarray(grid.depth),
                grid_wet_mask=np.asarray(grid.wet_mask),
                grid_wet_mask_3d=np.asarray(grid.wet_mask_3d))


def _digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    return h.hexdigest()


def _run_steps(step, state, nsteps):
    outs = []
    for _ in range(nsteps):
        state = step(state)
        outs.append(state)
    return outs


def make_step_case(name, nx, ny, nz, land_lat, physics, options, dt, dt_bt, restore_days,
                   nsteps, moving, seed=7):
    grid = workloads.build_grid(nx, ny, nz, land_lat=land_lat)
    T, S = workloads.initial_fields(grid, perturb_sigma=0.2)
    forcing = workloads.wind_forcing(grid)
    kw = dict(options)
    kw.update(forcing=forcing, dt_bt=dt_bt, dtype="float64")
    if restore_days > 0:
        kw.update(coastal_restore_mask=np.asarray(grid.wet_mask), coastal_restore_days=restore_days,
                  coastal_restore_T=_f32(T[:, :, 0]))
    step, init, _, params, _ = make_solver_global(grid, _physics(physics), dt, return_params=True, **kw)
    st = init(T_init=T, S_init=S)
    if moving:
        u, v, T0, S0, eta = _moving_state(grid, T, S, seed)
        st = JaxStateG(u, v, T0, S0, eta, np.zeros((nx, ny)))
    st = JaxStateG(*[_f32(a) for a in (st.u, st.v, st.T, st.S, st.eta)], np.zeros((nx, ny)))
    outs = _run_steps(step, st, nsteps)
    data = dict(_grid_arrays(grid))
    data.update(in_u=_np(st.u), in_v=_np(st.v), in_T=_np(st.T), in_S=_np(st.S), in_eta=_np(st.eta),
                dt=np.float64(dt), dt_bt=np.float64(dt_bt), restore_days=np.float64(restore_days),
                nsteps=np.int64(nsteps), n_subcyc=np.int64(params.n_subcyc),
                adv_nsub=np.int64(params.adv_nsub), conv_nsub=np.int64(params.conv_nsub),
                physics=np.array(repr(dataclasses.asdict(physics))),
                options=np.array(repr(options)))
    for n, s in enumerate(outs, start=1):
        if n == nsteps or (n == 1 and nsteps <= 2):
            for key in ("u", "v", "T", "S", "eta"):
                data[f"out{n}_{key}"] = _np(getattr(s, key))
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **data)
    print(name, "saved", {k: v.shape for k, v in data.items() if hasattr(v, 'shape') and v.ndim > 1})


def make_sponge_case(name="step_sponge_48x24x10", seed=7):
    """The step with the lateral sponge toward the initial fields and a
    mass-conserving eta relaxation box (factory.py:456-521, step.py:142-156,
    barotropic.py:22-41), strong enough to act within two steps."""
    nx, ny, nz = 48, 24, 10
    grid = workloads.build_grid(nx, ny, nz, land_lat=75.0)
    T, S = workloads.initial_fields(grid, perturb_sigma=0.2)
    lon, lat = np.asarray(grid.lon), np.asarray(grid.lat)
    extra = dict(sponge_days=0.5, sponge_cells=4, eta_relax_days=0.25,
                 eta_relax_box=(float(lon[10]), float(lon[20]), float(lat[8]), float(lat[14])), eta_relax_buffer=10.0)
    options = dict(workloads.PLAIN_OPTIONS, **extra)
    kw = dict(options, forcing=workloads.wind_forcing(grid), dt_bt=75.0, dtype="float64", T_init=T, S_init=S)
    step, init, _, params, _ = make_solver_global(grid, _physics(workloads.PLAIN_PHYSICS), 1800.0,
                                                  return_params=True, **kw)
    u, v, T0, S0, eta = _moving_state(grid, T, S, seed)
    st = JaxStateG(*[_f32(a) for a in (u, v, T0, S0, eta)], np.zeros((nx, ny)))
    outs = _run_steps(step, st, 2)
    data = dict(_grid_arrays(grid))
    data.update(in_u=_np(st.u), in_v=_np(st.v), in_T=_np(st.T), in_S=_np(st.S), in_eta=_np(st.eta),
                clim_T=_np(T), clim_S=_np(S), dt=np.float64(1800.0), dt_bt=np.float64(75.0),
                restore_days=np.float64(0.0), nsteps=np.int64(2), n_subcyc=np.int64(params.n_subcyc),
                adv_nsub=np.int64(params.adv_nsub), conv_nsub=np.int64(params.conv_nsub),
                physics=np.array(repr(dataclasses.asdict(workloads.PLAIN_PHYSICS))),
                options=np.array(repr(options)))
    for n, s in enumerate(outs, start=1):
        for key in ("u", "v", "T", "S", "eta"):
            data[f"out{n}_{key}"] = _np(getattr(s, key))
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **data)
    print(name, "saved")


def make_ledger_case(seed=9):
    """The reference's FP64 stage/source ledger (diagnostics/budgets.py:264-288
    ``make_budget_step``) over two steps with every source of the legacy path
    switched on: lateral sponge and eta relaxation, the column projection,
    bulk and coastal-bulk heat flux toward an air temperature, SSS restoring,
    coastal SST restoring and brine rejection below a raised freezing point."""
    from zhenmode.model.diagnostics.budgets import make_budget_step
    nx, ny, nz = 48, 24, 10
    grid = workloads.build_grid(nx, ny, nz, land_lat=75.0)
    T, S = workloads.initial_fields(grid, perturb_sigma=0.2)
    lon, lat = np.asarray(grid.lon), np.asarray(grid.lat)
    wm = np.asarray(grid.wet_mask)
    rng = np.random.default_rng(seed)
    coast = (wm * (rng.random((nx, ny)) < 0.3)).astype(np.float64)
    arrays = dict(T_atm=T[:, :, 0] - 2.0 + 0.5 * rng.standard_normal((nx, ny)),
                  S_ref_surf=S[:, :, 0] + 0.1 * rng.standard_normal((nx, ny)),
                  coastal_bulk_mask=coast, coastal_restore_mask=coast, coastal_restore_T=T[:, :, 0] + 1.0)
    scalars = dict(sponge_days=0.5, sponge_cells=4, eta_relax_days=0.25,
                   eta_relax_box=(float(lon[10]), float(lon[20]), float(lat[8]), float(lat[14])),
                   eta_relax_buffer=10.0, project_adv_vel=True, lambda_bulk=40.0, sss_restore_days=30.0,
                   coastal_bulk_lambda=20.0, coastal_restore_days=10.0, ice_salt_flux=2e-6, ice_freeze_temp_c=12.0)
    options = dict(workloads.PLAIN_OPTIONS, **scalars)
    tau_x, tau_y, _ = workloads.wind_forcing(grid)
    q_heat = np.broadcast_to((60.0 * np.cos(2.0 * np.radians(lat)))[None, :], (nx, ny)).copy()
    kw = dict(options, **arrays, forcing=(tau_x, tau_y, q_heat), dt_bt=75.0, dtype="float64",
              T_init=T, S_init=S)
    step, init, _, params, _ = make_solver_global(grid, _physics(workloads.PLAIN_PHYSICS), 1800.0,
                                                  return_params=True, **kw)
    advance = make_budget_step(params)
    u, v, T0, S0, eta = _moving_state(grid, T, S, seed)
    st = JaxStateG(*[_f32(a) for a in (u, v, T0, S0, eta)], np.zeros((nx, ny)))
    data = dict(_grid_arrays(grid))
    data.update(in_u=_np(st.u), in_v=_np(st.v), in_T=_np(st.T), in_S=_np(st.S), in_eta=_np(st.eta),
                clim_T=_np(T), clim_S=_np(S), dt=np.float64(1800.0), dt_bt=np.float64(75.0),
                restore_days=np.float64(0.0), nsteps=np.int64(2),
                physics=np.array(repr(dataclasses.asdict(workloads.PLAIN_PHYSICS))),
                options=np.array(repr(options)), forcing_q=q_heat,
                **{f"arr_{k}": np.asarray(v) for k, v in arrays.items()})
    for n in (1, 2):
        st, ledger = advance(st)
        for key in ("u", "v", "T", "S", "eta"):
            data[f"out{n}_{key}"] = _np(getattr(st, key))
        for key, value in ledger.items():
            data[f"ledger{n}_{key}"] = _np(value)
    np.savez_compressed(os.path.join(HERE, "ledger_48x24x10.npz"), **data)
    print("ledger saved")


def make_operator_case(seed=11):
    """Single-operator goldens on a 24x16x6 grid with land blocks and a wet
    polar band, random fields (reference functions called directly)."""
    nx, ny, nz = 24, 16, 6
    grid = workloads.build_grid(nx, ny, nz, land_lat=80.0)
    wm = np.array(grid.wet_mask_3d)
    wm[3:7, 6:9, :] = 0.0          # a land block
    wm[12:15, 3:6, 3:] = 0.0       # a shallow shelf (ghost levels)
    grid.wet_mask_3d = wm
    grid.wet_mask = wm[:, :, 0].copy()
    grid.ocean_mask = grid.wet_mask > 0.5
    grid.land_mask = ~grid.ocean_mask
    physics = workloads.PLAIN_PHYSICS
    T, S = workloads.initial_fields(grid, perturb_sigma=0.2)
    forcing = workloads.wind_forcing(grid)
    results = {}
    for limiter in ("fct", "monotone", "centered"):
        kw = dict(workloads.PLAIN_OPTIONS)
        kw.update(forcing=forcing, dt_bt=75.0, dtype="float64",
                  fct_adv=(limiter == "fct"), monotone_adv=(limiter == "monotone"),
                  coastal_restore_mask=np.asarray(grid.wet_mask), coastal_restore_days=30.0,
                  coastal_restore_T=_f32(T[:, :, 0]))
        _, _, _, p, _ = make_solver_global(grid, _physics(physics), 1800.0, return_params=True, **kw)
        u, v, T0, S0, eta = (_f32(a) for a in _moving_state(grid, T, S, seed, amp_u=0.2, amp_eta=0.3))
        st = JaxStateG(u, v, T0, S0, eta, np.zeros((nx, ny)))
        Fz = ref_transport._vertical_transport_iface(u, v, p)
        results[f"{limiter}_adv_T"] = _np(ref_transport._advection_scalar(T0, u, v, Fz, p))
        results[f"{limiter}_tracer_residual_T"], results[f"{limiter}_tracer_residual_S"] = (
            _np(a) for a in ref_tend._compute_tracer_residual(st, p))
        if limiter != "fct":
            continue
        results["Fz"] = _np(Fz)
        results["lap_u"] = _np(ref_h._laplacian_h(u, p))
        results["bih_u"] = _np(ref_h._biharmonic_h(u, p))
        results["hdiff_T"] = _np(ref_h._horizontal_tracer_diffusion(T0, p))
        results["bihT_T"] = _np(ref_h._horizontal_biharmonic_tracer(T0, p))
        results["d2z_T"] = _np(ref_v._d2_dz2(T0, p))
        results["ddz_u"] = _np(ref_v._d_dz(ref_v._fill_ghost_bottom(u, p), p))
        w = ref_transport._compute_vertical_velocity(st, p)
        ax, ay = ref_transport._advection_flux_form(u, v, w, p)
        results["madv_u"], results["madv_v"] = _np(ax), _np(ay)
        results["dealias_u"] = _np(ref_h._dealias_h_fd(u, p))
        gx, gy = ref_pressure._compute_pressure_gradient(st, p)
        results["pgf_x"], results["pgf_y"] = _np(gx), _np(gy)
        fx, fy = ref_pressure._compute_bt_rho_pgf(st, p)
        results["btrho_x"], results["btrho_y"] = _np(fx), _np(fy)
        col, unst = ref_pv._convective_mask(st, p)
        results["conv_T"] = _np(ref_pv._conv_flux_tendency(T0, col, p.kappa_conv, p, unst))
        mu, mv = ref_tend._compute_momentum_residual(st, p)
        results["mom_residual_u"], results["mom_residual_v"] = _np(mu), _np(mv)
        ubt, vbt = ref_transport._barotropic_velocity(u, v, p)
        results["ubt"], results["vbt"] = _np(ubt), _np(vbt)
        e1, u1, v1 = ref_bt._free_surface_step_fd(eta, ubt, vbt, p, fx, fy, dt_half=p.dt_bt)
        results["fs_eta"], results["fs_ubt"], results["fs_vbt"] = _np(e1), _np(u1), _np(v1)
        results["cap_T"] = _np(ref_h._apply_polar_cap(T0, p.wet_mask_z, p))
        results["cap_eta"] = _np(ref_h._apply_polar_cap(eta, p.wet_mask, p))
        lh = ref_step._linear_half_step(st, p, p.dt / 2)
        for key in ("u", "v", "T", "S"):
            results[f"lin_{key}"] = _np(getattr(lh, key))
        nl = ref_step._explicit_full_step(st, p, p.dt)
        for key in ("u", "v", "T", "S"):
            results[f"nl_{key}"] = _np(getattr(nl, key))
        results.update(in_u=u, in_v=v, in_T=T0, in_S=S0, in_eta=eta)
    data = dict(_grid_arrays(grid))
    data.update(results)
    np.savez_compressed(os.path.join(HERE, "operators_24x16x6.npz"), **data)
    print("operators saved", len(results), "arrays")


def make_diagnostics_case(seed=5):
    """The reference's diagnostics closure (factory.py:752-760: rho, hydrostatic
    pressure, vertical velocity), with and without a surface-pressure load, and
    its budget snapshot (diagnostics/snapshot.py:67-128) on a moving float32
    state of the 48x24x10 option-set grid."""
    from zhenmode.model.diagnostics import snapshot as ref_snapshot
    grid = workloads.build_grid(48, 24, 10, land_lat=75.0)
    T, S = workloads.initial_fields(grid, perturb_sigma=0.2)
    kw = dict(workloads.PLAIN_OPTIONS)
    kw.update(forcing=workloads.wind_forcing(grid), dt_bt=75.0, dtype="float64")
    _, _, diagnostics = make_solver_global(grid, _physics(workloads.PLAIN_PHYSICS), 1800.0, **kw)
    u, v, T0, S0, eta = _moving_state(grid, T, S, seed, amp_u=0.1, amp_eta=0.3)
    st = JaxStateG(*[_f32(a) for a in (u, v, T0, S0, eta)], np.zeros((48, 24)))
    rng = np.random.default_rng(seed + 1)
    sp = _f32(101325.0 + 500.0 * _smooth_noise(rng, (48, 24)))
    rho, pres, w = diagnostics(st)
    _, pres_sp, _ = diagnostics(st, surface_pressure_pa=sp)
    b = ref_snapshot.compute_budget_diagnostics(st, grid)
    data = dict(_grid_arrays(grid))
    data.update(in_u=_np(st.u), in_v=_np(st.v), in_T=_np(st.T), in_S=_np(st.S), in_eta=_np(st.eta),
                surface_pressure_pa=sp, rho=_np(rho), pressure=_np(pres), w=_np(w), pressure_sp=_np(pres_sp),
                budget_names=np.array(list(b.as_dict().keys())),
                budget_values=np.array(list(b.as_dict().values()), dtype=np.float64),
                options=np.array(repr(workloads.PLAIN_OPTIONS)))
    np.savez_compressed(os.path.join(HERE, "diagnostics_48x24x10.npz"), **data)
    print("diagnostics saved", dict(zip(b.as_dict().keys(), b.as_dict().values())))


def make_seasonal_case(seed=9):
    """The reference's seasonal blend (inputs/forcing/seasonal.py:86-103) of a
    random 12-month stack at days around the month boundaries."""
    from zhenmode.model.inputs.forcing import seasonal as ref_seasonal
    stack = _f32(np.random.default_rng(seed).standard_normal((12, 8, 6)))
    days = np.array([0.0, 1.0, 2.4, 14.5, 27.6, 28.7, 29.9, 30.0, 31.2, 359.5, 361.0, 725.3])
    out = np.stack([_np(ref_seasonal.interp_monthly_field_jit(stack, float(d), 5.0)) for d in days])
    out0 = np.stack([_np(ref_seasonal.interp_monthly_field_jit(stack, float(d), 0.0)) for d in days])
    np.savez_compressed(os.path.join(HERE, "seasonal_blend.npz"), stack=stack, days=days, blend5=out, blend0=out0)
    print("seasonal saved")


def make_projection_case(seed=13):
    """The reference's column-divergence projection (dynamics/projection.py:64-127)
    called on a moving float64 state of the 48x24x10 option-set grid, with
    the preset's settings and with the Jacobi preconditioner."""
    from zhenmode.model.solver.dynamics import projection as ref_proj
    grid = workloads.build_grid(48, 24, 10, land_lat=75.0)
    T, S = workloads.initial_fields(grid, perturb_sigma=0.2)
    data = dict(_grid_arrays(grid))
    u, v, T0, S0, eta = _moving_state(grid, T, S, seed, amp_u=0.2)
    data.update(in_u=_f32(u), in_v=_f32(v))
    for pre in ("none", "jacobi"):
        kw = dict(workloads.PLAIN_OPTIONS)
        kw.update(forcing=workloads.wind_forcing(grid), dt_bt=75.0, dtype="float64", project_adv_vel=True,
                  projection_preconditioner=pre)
        _, _, _, params, _ = make_solver_global(grid, _physics(workloads.PLAIN_PHYSICS), 1800.0,
                                                return_params=True, **kw)
        ua, va = ref_proj._project_column_divergence(_f32(u), _f32(v), params, 1800.0)
        data[f"{pre}_u"] = _np(ua)
        data[f"{pre}_v"] = _np(va)
    np.savez_compressed(os.path.join(HERE, "projection_48x24x10.npz"), **data)
    print("projection saved")


def make_terms_case(seed=17):
    """The reference's tracer-term decomposition (``terms_fn`` of
    factory.py:762-764, dynamics/tendencies.py:74-92) on a moving float32
    state of the 48x24x10 option-set grid with cold surface patches, so that
    convection acts."""
    grid = workloads.build_grid(48, 24, 10, land_lat=75.0)
    T, S = workloads.initial_fields(grid, perturb_sigma=0.2)
    kw = dict(workloads.PLAIN_OPTIONS)
    kw.update(forcing=workloads.wind_forcing(grid), dt_bt=75.0, dtype="float64", return_params=True,
              coastal_kappa_h_mask=np.asarray(grid.wet_mask), coastal_kappa_h=50.0,
              coastal_kappa_v_mask=np.asarray(grid.wet_mask), coastal_kappa_v=2e-5)
    out = make_solver_global(grid, _physics(workloads.PLAIN_PHYSICS), 1800.0, **kw)
    terms_fn = out[4]
    u, v, T0, S0, eta = _moving_state(grid, T, S, seed, amp_u=0.1, amp_eta=0.3)
    rng = np.random.default_rng(seed + 1)
    cold = (_smooth_noise(rng, (48, 24)) > 1.0) * np.asarray(grid.wet_mask)
    T0 = T0.copy()
    T0[:, :, :2] -= 4.0 * cold[:, :, None]
    st = JaxStateG(*[_f32(a) for a in (u, v, T0, S0, eta)], np.zeros((48, 24)))
    terms = terms_fn(st)
    data = dict(_grid_arrays(grid))
    data.update(in_u=_np(st.u), in_v=_np(st.v), in_T=_np(st.T), in_S=_np(st.S), in_eta=_np(st.eta),
                coastal_kappa_h=np.float64(50.0), coastal_kappa_v=np.float64(2e-5),
                terms=_np(terms), options=np.array(repr(workloads.PLAIN_OPTIONS)))
    np.savez_compressed(os.path.join(HERE, "terms_48x24x10.npz"), **data)
    print("terms saved", [float(np.abs(t).max()) for t in _np(terms)])


def make_mld_case(seed=19):
    """The reference's density-threshold mixed-layer depth
    (diagnostics/mixed_layer.py:39-74) of perturbed thermocline columns with
    the levels below the seafloor missing (NaN)."""
    from zhenmode.model.diagnostics.mixed_layer import mixed_layer_depth
    grid = workloads.build_grid(24, 16, 20, land_lat=70.0)
    T, S = workloads.initial_fields(grid, perturb_sigma=0.2)
    rng = np.random.default_rng(seed)
    T = T + 0.3 * rng.standard_normal(T.shape)
    wet3 = np.asarray(grid.wet_mask_3d)
    mld = mixed_layer_depth(np.where(wet3 > 0.5, T, np.nan), np.where(wet3 > 0.5, S, np.nan), np.asarray(grid.z),
                            ocean=np.asarray(grid.wet_mask) > 0.5)
    np.savez_compressed(os.path.join(HERE, "mld_24x16x20.npz"), T=T, S=S, z=np.asarray(grid.z), wet3=wet3, mld=mld)
    print("mld saved", np.nanmin(mld), np.nanmax(mld))


def main():
    make_terms_case()
    make_mld_case()
    make_ledger_case()
    make_sponge_case()
    make_operator_case()
    make_projection_case()
    make_seasonal_case()
    make_diagnostics_case()
    # The 0.5 deg production option set, rescaled to a 7.5 deg x 7.5 deg grid
    # whose polar bands are partly wet, from a moving state (2 steps).
    make_step_case("step_plain_48x24x10", 48, 24, 10, 75.0, workloads.PLAIN_PHYSICS,
                   workloads.PLAIN_OPTIONS, 1800.0, 75.0, 30.0, 2, moving=True)
    # The 0.5 deg preset proper: column projection of the stage-2 advective
    # velocity on (dynamics/projection.py, step.py:292-303).
    make_step_case("step_projected_48x24x10", 48, 24, 10, 75.0, workloads.PLAIN_PHYSICS,
                   dict(workloads.PLAIN_OPTIONS, project_adv_vel=True), 1800.0, 75.0, 30.0, 2, moving=True)
    # Same physics from rest on an all-land-polar grid (production geometry).
    make_step_case("step_plain_rest_64x32x12", 64, 32, 12, 65.0, workloads.PLAIN_PHYSICS,
                   workloads.PLAIN_OPTIONS, 1800.0, 75.0, 30.0, 1, moving=False)
    # The CPU-runnable smoke configuration: 90x45x15, float64, 8 steps of 10 s.
    wl = workloads.WORKLOADS["smoke"]
    make_step_case("step_smoke_90x45x15", wl.nx, wl.ny, wl.nz, 65.0, wl.physics, wl.options,
                   wl.dt, wl.dt_bt, 0.0, wl.steps, moving=False)


if __name__ == "__main__":
    main()
