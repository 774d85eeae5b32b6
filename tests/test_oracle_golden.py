"""Pin the float64 oracle to golden vectors produced by ZhenMode's own step code.

The fixtures come from ``tests/golden/make_golden.py`` (the reference solver
run unmodified, float64).  Agreement is at round-off level: the oracle is a
restatement of the same arithmetic, so anything above ~1e-12 relative is a
transcription error, not precision.
"""
import numpy as np
import pytest

from oracle import params as oparams
from oracle import step as ostep
from tests.golden_io import case_inputs, grid_from, load, rel_l2

TOL = 1e-11


def _operator_params(data, limiter):
    from zhenmode_b200 import workloads
    grid = grid_from(data)
    T = data["in_T"]
    kw = dict(workloads.PLAIN_OPTIONS)
    lat = np.radians(np.asarray(grid.lat))
    tau_x = np.broadcast_to((0.1 * np.sin(2 * lat) * np.cos(lat))[None, :], (grid.nx, grid.ny)).copy()
    zeros = np.zeros((grid.nx, grid.ny))
    kw.update(forcing=(tau_x, zeros, zeros.copy()), dt_bt=75.0, dtype="float64",
              fct_adv=(limiter == "fct"), monotone_adv=(limiter == "monotone"),
              coastal_restore_mask=np.asarray(grid.wet_mask), coastal_restore_days=30.0,
              coastal_restore_T=np.array(T[:, :, 0]))
    return oparams.build_params(grid, workloads.PLAIN_PHYSICS, 1800.0, **kw)


@pytest.fixture(scope="module")
def ops():
    return load("operators_24x16x6")


def _check(name, got, want, tol=TOL):
    err = rel_l2(got, want)
    assert err < tol, f"{name}: rel L2 {err:.3e}"


@pytest.mark.parametrize("limiter", ["fct", "monotone", "centered"])
def test_tracer_advection_and_residual(ops, limiter):
    p = _operator_params(ops, limiter)
    u, v, T, S = ops["in_u"], ops["in_v"], ops["in_T"], ops["in_S"]
    Fz = ostep.vertical_transport_iface(u, v, p)
    _check("adv_T", ostep.tracer_advection(T, u, v, Fz, p), ops[f"{limiter}_adv_T"])
    rT, rS = ostep.tracer_residual(u, v, T, S, p)
    _check("res_T", rT, ops[f"{limiter}_tracer_residual_T"])
    _check("res_S", rS, ops[f"{limiter}_tracer_residual_S"])


def test_single_operators(ops):
    p = _operator_params(ops, "fct")
    u, v, T, S, eta = (ops["in_" + k] for k in ("u", "v", "T", "S", "eta"))
    _check("Fz", ostep.vertical_transport_iface(u, v, p), ops["Fz"])
    _check("lap", ostep.laplacian_h(u, p), ops["lap_u"])
    _check("bih", ostep.biharmonic_h(u, p), ops["bih_u"])
    _check("hdiff", ostep.horizontal_tracer_diffusion(T, p), ops["hdiff_T"])
    _check("bihT", ostep.horizontal_biharmonic_tracer(T, p), ops["bihT_T"])
    _check("d2z", ostep.d2_dz2(T, p), ops["d2z_T"])
    _check("ddz", ostep.d_dz(ostep.fill_ghost_bottom(u, p), p), ops["ddz_u"])
    w = ostep.vertical_velocity(u, v, p)
    ax, ay = ostep.momentum_advection(u, v, w, p)
    _check("madv_u", ax, ops["madv_u"])
    _check("madv_v", ay, ops["madv_v"])
    _check("dealias", ostep.dealias(u, p), ops["dealias_u"])
    gx, gy = ostep.pressure_gradient(T, S, eta, p)
    _check("pgf_x", gx, ops["pgf_x"])
    _check("pgf_y", gy, ops["pgf_y"])
    fx, fy = ostep.bt_rho_pgf(T, S, p)
    _check("btrho_x", fx, ops["btrho_x"])
    _check("btrho_y", fy, ops["btrho_y"])
    col, unst = ostep.convective_gates(T, S, p)
    _check("conv", ostep.convective_tendency(T, col, p.kappa_conv, p, unst), ops["conv_T"])
    mu, mv = ostep.momentum_residual(u, v, T, S, eta, p)
    _check("mres_u", mu, ops["mom_residual_u"])
    _check("mres_v", mv, ops["mom_residual_v"])
    ubt, vbt = ostep.barotropic_velocity(u, v, p)
    _check("ubt", ubt, ops["ubt"])
    _check("vbt", vbt, ops["vbt"])
    e1, u1, v1 = ostep.free_surface_step(eta, ubt, vbt, p, fx, fy, p.dt_bt)
    _check("fs_eta", e1, ops["fs_eta"])
    _check("fs_ubt", u1, ops["fs_ubt"])
    _check("fs_vbt", v1, ops["fs_vbt"])
    _check("cap_T", ostep.polar_cap(T, p.wet_mask_z, p), ops["cap_T"])
    _check("cap_eta", ostep.polar_cap(eta, p.wet_mask, p), ops["cap_eta"])
    st = dict(u=u, v=v, T=T, S=S, eta=eta)
    lh = ostep.linear_half_step(st, p, p.dt / 2)
    for k in ("u", "v", "T", "S"):
        _check("lin_" + k, lh[k], ops["lin_" + k])
    nl = ostep.explicit_full_step(st, p)
    for k in ("u", "v", "T", "S"):
        _check("nl_" + k, nl[k], ops["nl_" + k])


@pytest.mark.parametrize("name", ["step_plain_48x24x10", "step_projected_48x24x10", "step_sponge_48x24x10",
                                  "step_plain_rest_64x32x12", "step_smoke_90x45x15"])
def test_full_step(name):
    data = load(name)
    grid, physics, dt, options, state = case_inputs(data)
    p = oparams.build_params(grid, physics, dt, **options)
    assert p.n_subcyc == int(data["n_subcyc"])
    assert p.adv_nsub == int(data["adv_nsub"])
    assert p.conv_nsub == int(data["conv_nsub"])
    st = {k: np.array(v) for k, v in state.items()}
    nsteps = int(data["nsteps"])
    for n in range(1, nsteps + 1):
        st = ostep.step(st, p)
        if f"out{n}_u" in data:
            for k in ("u", "v", "T", "S", "eta"):
                want = data[f"out{n}_{k}"]
                if np.linalg.norm(want) == 0:
                    assert np.max(np.abs(st[k])) < 1e-14
                else:
                    _check(f"{name} step {n} {k}", st[k], want, tol=1e-10)


def _diag_case():
    from zhenmode_b200 import workloads
    data = load("diagnostics_48x24x10")
    grid = grid_from(data)
    lat = np.radians(np.asarray(grid.lat))
    tau_x = np.broadcast_to((0.1 * np.sin(2 * lat) * np.cos(lat))[None, :], (grid.nx, grid.ny)).copy()
    zeros = np.zeros((grid.nx, grid.ny))
    kw = dict(workloads.PLAIN_OPTIONS)
    kw.update(forcing=(tau_x, zeros, zeros.copy()), dt_bt=75.0, dtype="float64")
    p = oparams.build_params(grid, workloads.PLAIN_PHYSICS, 1800.0, **kw)
    state = {k: data["in_" + k] for k in ("u", "v", "T", "S", "eta")}
    return data, grid, p, state


def test_diagnostics_closure():
    """rho, hydrostatic pressure (with and without a surface load) and the
    vertical velocity of the reference's diagnostics closure."""
    data, grid, p, state = _diag_case()
    rho, pres, w = ostep.diagnostics(state, p)
    _check("rho", rho, data["rho"])
    _check("pressure", pres, data["pressure"])
    _check("w", w, data["w"])
    _, pres_sp, _ = ostep.diagnostics(state, p, surface_pressure_pa=data["surface_pressure_pa"])
    _check("pressure_sp", pres_sp, data["pressure_sp"])


def test_budget_diagnostics():
    from oracle import budgets
    data, grid, p, state = _diag_case()
    got = budgets.budget_diagnostics(state["T"], state["S"], grid.dx_2d, grid.dy, grid.z, grid.wet_mask,
                                     grid.wet_mask_3d)
    names = [str(n) for n in data["budget_names"]]
    assert names == list(budgets.FIELDS)
    for name, want in zip(names, data["budget_values"]):
        assert abs(got[name] - want) <= 1e-13 * abs(want), (name, got[name], want)


def test_seasonal_blend():
    from oracle import seasonal
    data = load("seasonal_blend")
    for n, day in enumerate(data["days"]):
        _check(f"blend5 day {day}", seasonal.blend(data["stack"], float(day), 5.0), data["blend5"][n], 1e-14)
        _check(f"blend0 day {day}", seasonal.blend(data["stack"], float(day), 0.0), data["blend0"][n], 1e-14)


@pytest.mark.parametrize("pre", ["none", "jacobi"])
def test_column_projection(pre):
    from zhenmode_b200 import workloads
    data = load("projection_48x24x10")
    grid = grid_from(data)
    kw = dict(workloads.PLAIN_OPTIONS)
    kw.update(forcing=workloads.wind_forcing(grid), dt_bt=75.0, dtype="float64", project_adv_vel=True,
              projection_preconditioner=pre)
    p = oparams.build_params(grid, workloads.PLAIN_PHYSICS, 1800.0, **kw)
    ua, va = ostep.project_column_divergence(data["in_u"], data["in_v"], p, 1800.0)
    _check("u", ua, data[f"{pre}_u"], 1e-9)
    _check("v", va, data[f"{pre}_v"], 1e-9)


def test_ledger_matches_reference_budget_step():
    """The FP64 stage/source ledger (diagnostics/budgets.py:264-288) of two
    steps with every legacy source on, against the reference's own
    make_budget_step."""
    from oracle import ledger
    data = load("ledger_48x24x10")
    grid, physics, dt, options, state = case_inputs(data)
    p = oparams.build_params(grid, physics, dt, **options)
    st = {k: np.array(v) for k, v in state.items()}
    for n in (1, 2):
        st, led = ledger.ledger_step(st, p)
        for k in ("u", "v", "T", "S", "eta"):
            _check(f"step {n} {k}", st[k], data[f"out{n}_{k}"], tol=1e-10)
        for key, value in led.items():
            want = data[f"ledger{n}_{key}"]
            got = np.asarray(value, dtype=np.float64)
            assert got.shape == want.shape, key
            scale = max(float(np.max(np.abs(want))), 1e-300)
            err = float(np.max(np.abs(got - want))) if got.size else 0.0
            # residual identities are differences of large sums: compared with the sums they close
            if "residual" in key:
                ref = {"decomposition_residual": "change_scale", "absolute_decomposition_residual": "change_scale",
                       "budget_residual": "change_scale", "absolute_budget_residual": "change_scale",
                       "advection_boundary_residual": "nonlinear_process_scale",
                       "absolute_advection_boundary_residual": "nonlinear_process_scale",
                       "nonlinear_accounting_residual": "nonlinear_process_scale",
                       "absolute_nonlinear_accounting_residual": "nonlinear_process_scale"}.get(key)
                if ref is not None:
                    scale = max(scale, float(np.max(np.abs(data[f"ledger{n}_{ref}"]))))
            assert err <= 1e-9 * scale, (n, key, err, scale)


def _terms_case():
    from zhenmode_b200 import workloads
    data = load("terms_48x24x10")
    grid = grid_from(data)
    wm = np.asarray(grid.wet_mask)
    kw = dict(workloads.PLAIN_OPTIONS)
    kw.update(forcing=workloads.wind_forcing(grid), dt_bt=75.0,
              coastal_kappa_h_mask=wm, coastal_kappa_h=float(data["coastal_kappa_h"]),
              coastal_kappa_v_mask=wm, coastal_kappa_v=float(data["coastal_kappa_v"]))
    state = {k: data["in_" + k] for k in ("u", "v", "T", "S", "eta")}
    return data, grid, kw, state


def test_tracer_terms_match_reference_terms_fn():
    """terms_fn of factory.py:762-764 (dynamics/tendencies.py:74-92)."""
    from zhenmode_b200 import workloads
    data, grid, kw, state = _terms_case()
    p = oparams.build_params(grid, workloads.PLAIN_PHYSICS, 1800.0, dtype="float64", **kw)
    got = ostep.tracer_terms(state, p)
    want = data["terms"]
    assert got.shape == want.shape == (6,) + state["T"].shape
    assert np.abs(want[3]).max() > 0, "the fixture must exercise convection"
    for n, name in enumerate(("adv", "diff_h", "diff_v", "conv", "gm", "redi")):
        if np.abs(want[n]).max() == 0:
            assert np.abs(got[n]).max() == 0, name
        else:
            _check(name, got[n], want[n])
