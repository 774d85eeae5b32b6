"""Parity of the CUDA step (float32 fields, float64 barotropic mode) with the
float64 oracle and with golden vectors of the reference's own step code.

All calls go through the C ABI (``zm_run_stage`` / ``zm_step``).  The
tolerances are relative L2 norms per field; one production step is held to
1e-5.
"""
import numpy as np
import pytest

from oracle import step as ostep
from tests import gpu_util as gu
from tests.golden_io import case_inputs, grid_from, load
from zhenmode_b200 import workloads

pytestmark = pytest.mark.gpu

STEP_TOL = 1e-5          # one step, every field
STAGE_TOL = 1e-5         # one stage on a moving state


def _operator_case():
    data = load("operators_24x16x6")
    grid = grid_from(data)
    T = data["in_T"]
    kw = dict(workloads.PLAIN_OPTIONS)
    lat = np.radians(np.asarray(grid.lat))
    tau_x = np.broadcast_to((0.1 * np.sin(2 * lat) * np.cos(lat))[None, :], (grid.nx, grid.ny)).copy()
    zeros = np.zeros((grid.nx, grid.ny))
    kw.update(forcing=(tau_x, zeros, zeros.copy()), dt_bt=75.0,
              coastal_restore_mask=np.asarray(grid.wet_mask), coastal_restore_days=30.0,
              coastal_restore_T=np.array(T[:, :, 0]))
    state = {k: data["in_" + k] for k in gu.FIELDS}
    return grid, workloads.PLAIN_PHYSICS, 1800.0, kw, state


@pytest.fixture(scope="module")
def operator_case():
    grid, physics, dt, kw, state = _operator_case()
    gpu, p = gu.build_pair(grid, physics, dt, kw)
    return gpu, p, state


def test_linear_half_step_matches_oracle(operator_case):
    gpu, p, state = operator_case
    got = gu.run_stage(gpu, 1, state)
    want = ostep.linear_half_step(dict(state), p, p.dt / 2)
    errs = gu.errors(got, want, ("u", "v", "T", "S"))
    assert max(errs.values()) < STAGE_TOL, errs


def test_nonlinear_step_matches_oracle(operator_case):
    gpu, p, state = operator_case
    got = gu.run_stage(gpu, 2, state)
    want = ostep.explicit_full_step(dict(state), p)
    errs = gu.errors(got, want, ("u", "v", "T", "S"))
    assert max(errs.values()) < STAGE_TOL, errs


@pytest.mark.parametrize("limiter", ["monotone", "centered"])
def test_nonlinear_step_with_other_tracer_limiters(limiter):
    """The donor-cell (monotone_adv) and centred tracer face values
    (transport.py:199-290) in the N stage, against the oracle."""
    grid, physics, dt, kw, state = _operator_case()
    kw = dict(kw, fct_adv=False, monotone_adv=(limiter == "monotone"))
    gpu, p = gu.build_pair(grid, physics, dt, kw)
    got = gu.run_stage(gpu, 2, state)
    want = ostep.explicit_full_step(dict(state), p)
    errs = gu.errors(got, want, ("u", "v", "T", "S"))
    assert max(errs.values()) < STAGE_TOL, errs


def test_full_step_matches_oracle_on_moving_state(operator_case):
    gpu, p, state = operator_case
    got = gu.run_stage(gpu, 3, state)
    want = ostep.step(dict(state), p)
    errs = gu.errors(got, want)
    assert max(errs.values()) < STEP_TOL, errs


@pytest.mark.parametrize("name", ["step_plain_48x24x10", "step_sponge_48x24x10", "step_plain_rest_64x32x12",
                                  "step_smoke_90x45x15"])
def test_steps_match_reference_goldens(name):
    data = load(name)
    grid, physics, dt, options, state = case_inputs(data)
    gpu, _ = gu.build_pair(grid, physics, dt, options)
    nsteps = int(data["nsteps"])
    got = gu.run_steps(gpu, state, 1)
    want = {k: data[f"out1_{k}"] for k in gu.FIELDS} if "out1_u" in data else None
    if want is not None:
        errs = gu.errors(got, want)
        assert max(errs.values()) < STEP_TOL, errs
    got_n = gu.run_steps(gpu, state, nsteps)
    want_n = {k: data[f"out{nsteps}_{k}"] for k in gu.FIELDS}
    errs = gu.errors(got_n, want_n)
    print(name, nsteps, "steps, relative L2:", errs)
    # Each step rounds the state to float32 and adds at most STEP_TOL against the
    # float64 reference; over n steps the differences add at most linearly.
    assert max(errs.values()) < nsteps * STEP_TOL, errs


def test_production_options_at_reduced_size():
    """The 0.5-degree option set on a 180x90x50 grid: one step from rest and
    from a 2-step spun-up state, against the oracle."""
    grid, physics, dt, kw, T, S = workloads.make_case("plain", 180, 90, 50, dtype="float32")
    gpu, p = gu.build_pair(grid, physics, dt, kw)
    from oracle.params import init_state
    st0 = gu.f32(init_state(p, T, S))
    want1 = ostep.step(dict(st0), p)
    got1 = gu.run_steps(gpu, st0, 1)
    errs = gu.errors(got1, want1)
    assert max(errs.values()) < STEP_TOL, errs
    start = gu.f32(want1)
    want2 = ostep.step(dict(start), p)
    got2 = gu.run_steps(gpu, start, 1)
    errs = gu.errors(got2, want2)
    assert max(errs.values()) < STEP_TOL, errs


def test_implicit_vertical_diffusion_matches_oracle():
    grid, physics, dt, kw, state = _operator_case()
    kw = dict(kw, vertical_diffusion="implicit")
    gpu, p = gu.build_pair(grid, physics, dt, kw)
    got = gu.run_stage(gpu, 1, state)
    want = ostep.linear_half_step(dict(state), p, p.dt / 2)
    errs = gu.errors(got, want, ("u", "v", "T", "S"))
    assert max(errs.values()) < STAGE_TOL, errs


def _moving(p, T, S, seed=5, amp=0.1):
    rng = np.random.default_rng(seed)
    from oracle.params import init_state
    st = gu.f32(init_state(p, T, S))
    wm = p.wet_mask_z
    st["u"] = gu.f32({k: amp * rng.standard_normal(wm.shape) * wm for k in gu.FIELDS})["u"]
    st["v"] = gu.f32({k: amp * rng.standard_normal(wm.shape) * wm for k in gu.FIELDS})["v"]
    st["v"][:, 0] = 0.0
    st["v"][:, -1] = 0.0
    return st


@pytest.mark.parametrize("shape", [(24, 16, 6), (90, 45, 15), (180, 24, 10), (360, 20, 6), (720, 16, 4),
                                   (800, 12, 4)])
def test_momentum_advection_part_matches_oracle(shape):
    """Dealiased advection + wind part of the momentum residual (stage 4),
    including grids whose longitude mask drops the +-nx/3 bins; widths 180,
    360, 720 and 800 take the register-resident filter, 24 and 90 the
    shared-memory one."""
    from oracle.params import RHO_0
    grid, physics, dt, kw, T, S = workloads.make_case("plain", *shape, dtype="float32")
    gpu, p = gu.build_pair(grid, physics, dt, kw)
    st = _moving(p, T, S)
    w = ostep.vertical_velocity(st["u"], st["v"], p)
    ax, ay = ostep.momentum_advection(st["u"], st["v"], w, p)
    wind = lambda tau: (tau[:, :, None] * p.surface_mask / (RHO_0 * p.dz_surface)
                        - (tau / (RHO_0 * p.H_sw))[:, :, None]) * p.wet_mask_z
    got = gu.run_stage(gpu, 4, st)
    err_u = gu.rel_l2(got["u"] - wind(p.tau_x_2d), ax)
    err_v = gu.rel_l2(got["v"] - wind(p.tau_y_2d), ay)
    assert max(err_u, err_v) < 1e-5, (err_u, err_v)


@pytest.mark.parametrize("shape", [(24, 16, 6), (90, 45, 15)])
def test_pressure_part_matches_oracle(shape):
    """Baroclinic pressure-gradient force minus its barotropic layer mean (stage 5)."""
    from oracle.params import RHO_0
    grid, physics, dt, kw, T, S = workloads.make_case("plain", *shape, dtype="float32")
    gpu, p = gu.build_pair(grid, physics, dt, kw)
    st = _moving(p, T, S)
    gx, gy = ostep.gradient_conservative_3d(ostep.baroclinic_pressure(st["T"], st["S"], p), p)
    fx, fy = ostep.bt_rho_pgf(st["T"], st["S"], p)
    got = gu.run_stage(gpu, 5, st)
    err_u = gu.rel_l2(got["u"], (-gx / RHO_0 - fx[:, :, None]) * p.wet_mask_z)
    err_v = gu.rel_l2(got["v"], (-gy / RHO_0 - fy[:, :, None]) * p.wet_mask_z)
    assert max(err_u, err_v) < 1e-5, (err_u, err_v)



def _polar_case(nx, ny, nz, land_lat, barotropic_kernel="auto", **extra):
    """The 0.5-degree option set on a grid whose polar cap band rows are all
    land (land_lat = 65: the barotropic polar cap is the identity) or partly
    ocean (land_lat = 87 on a 1.9-degree grid: the cap averages wet band
    rows), with a moving state."""
    wl = workloads.WORKLOADS["plain"]
    grid = workloads.build_grid(nx, ny, nz, land_lat=land_lat)
    T, S = workloads.initial_fields(grid, perturb_sigma=wl.perturb_sigma)
    kw = dict(wl.options)
    kw.update(forcing=workloads.wind_forcing(grid), dt_bt=wl.dt_bt,
              coastal_restore_mask=np.asarray(grid.wet_mask), coastal_restore_days=wl.restore_days,
              coastal_restore_T=np.array(T[:, :, 0]), barotropic_kernel=barotropic_kernel)
    if extra.pop("sponge_targets", False):
        kw.update(T_init=T, S_init=S)
    kw.update(extra)
    gpu, p = gu.build_pair(grid, wl.physics, wl.dt, kw)
    from oracle.params import init_state
    st = init_state(p, T, S)
    lon = np.radians(np.asarray(grid.lon))[:, None, None]
    lat = np.radians(np.asarray(grid.lat))[None, :, None]
    wet3 = np.asarray(grid.wet_mask_3d)
    st["u"] = 0.1 * np.cos(lat) * np.sin(3 * lon) * wet3
    st["v"] = 0.05 * np.sin(2 * lon) * np.cos(lat) ** 2 * wet3
    st["eta"] = 0.2 * np.sin(lon[:, :, 0]) * np.cos(lat[:, :, 0]) * np.asarray(grid.wet_mask)
    return gpu, p, gu.f32(st)


@pytest.mark.parametrize("land_lat,kernel,resident,cap", [
    (87.0, "auto", True, True),          # resident tiles, cap active
    (87.0, "streaming", False, True),    # streaming kernels, cap active
    (65.0, "streaming", False, False),   # streaming kernels, cap the identity
])
def test_barotropic_paths_match_oracle(land_lat, kernel, resident, cap):
    gpu, p, st = _polar_case(192, 96, 8, land_lat, kernel)
    solver = gpu.solver
    assert (solver.bt_blocks > 0) == resident
    assert bool(solver.bt_cap_active) == cap
    want = ostep.step(dict(st), p)
    got = gu.run_steps(gpu, st, 1)
    errs = gu.errors(got, want)
    assert max(errs.values()) < STEP_TOL, errs


@pytest.mark.parametrize("kernel,resident", [("auto", True), ("streaming", False)])
def test_sponge_and_eta_relaxation_match_oracle(kernel, resident):
    """Lateral sponge toward the initial fields in the L half steps and on the
    barotropic mode, and an eta relaxation box, each with the uniform refill
    of the removed volume (barotropic.py:22-41), on both barotropic paths."""
    grid_lon = np.linspace(-180.0, 180.0, 192, endpoint=False)
    gpu, p, st = _polar_case(192, 96, 8, 87.0, kernel, sponge_targets=True, sponge_days=0.5, sponge_cells=6,
                             eta_relax_days=0.25, eta_relax_box=(float(grid_lon[40]), float(grid_lon[70]), 10.0, 30.0),
                             eta_relax_buffer=6.0)
    assert (gpu.solver.bt_blocks > 0) == resident
    want = ostep.step(dict(st), p)
    got = gu.run_steps(gpu, st, 1)
    errs = gu.errors(got, want)
    assert max(errs.values()) < STEP_TOL, errs


def test_barotropic_kernel_choice_follows_grid_size():
    """More tiles than the GPU holds at once: 'auto' streams, 'resident' is refused."""
    from zhenmode_b200 import UnsupportedOption, make_solver_global
    wl = workloads.WORKLOADS["plain"]
    grid = workloads.build_grid(2048, 1024, 3)
    kw = dict(wl.options, dt_bt=wl.dt_bt, dtype="float32")
    step = make_solver_global(grid, wl.physics, wl.dt, **kw)[0]
    assert step.solver.bt_blocks == 0
    with pytest.raises(UnsupportedOption):
        make_solver_global(grid, wl.physics, wl.dt, barotropic_kernel="resident", **kw)


def test_deepest_grid_matches_oracle():
    """nz = 64, the limit of the one-word-per-column wet mask (bit 63 wet at
    the deep columns), one step of the 0.5-degree option set on a moving state."""
    grid, physics, dt, kw, T, S = workloads.make_case("plain", 24, 16, 64, dtype="float32")
    kw = {k: v for k, v in kw.items() if k != "dtype"}
    gpu, p = gu.build_pair(grid, physics, dt, kw)
    assert int(np.asarray(grid.wet_mask_3d)[:, :, 63].sum()) > 0
    from oracle.params import init_state
    st = init_state(p, T, S)
    wet3 = np.asarray(grid.wet_mask_3d)
    lat = np.radians(np.asarray(grid.lat))[None, :, None]
    st["u"] = 0.1 * np.cos(lat) * wet3
    st["v"] = 0.02 * np.sin(2 * lat) * wet3
    st = gu.f32(st)
    want = ostep.step(dict(st), p)
    got = gu.run_steps(gpu, st, 1)
    errs = gu.errors(got, want)
    assert max(errs.values()) < STEP_TOL, errs


def test_longitude_sizes_outside_2_3_5_are_refused():
    """The longitude filter's FFT takes nx = 2^a 3^b 5^c (zm_create: ZM_ERR_UNSUPPORTED)."""
    from zhenmode_b200 import UnsupportedOption, make_solver_global
    grid, physics, dt, kw, _, _ = workloads.make_case("plain", 28, 16, 8, dtype="float32")
    with pytest.raises(UnsupportedOption):
        make_solver_global(grid, physics, dt, **kw)
