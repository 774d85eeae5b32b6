"""Column-divergence projection of the stage-2 advective velocity
(dynamics/projection.py:10-127, timestepping/step.py:292-303) on the GPU.

Stage 8 of ``zm_run_stage`` applies the projection alone.  The GPU runs the
float32 mode, whose CG tolerances have the float32 floors
(tol = transport rtol = 32 eps = 3.8e-6, factory.py:385-386); the oracle is
run in float64 arithmetic with those same tolerances for the tight
comparison, and the reference's float64 goldens (tolerance 1e-12) bound the
gap that the looser stopping rule leaves.
"""
import numpy as np
import pytest

from oracle import params as oparams
from oracle import step as ostep
from tests import gpu_util as gu
from tests.golden_io import case_inputs, grid_from, load, rel_l2
from zhenmode_b200 import make_solver_global, workloads

pytestmark = pytest.mark.gpu

TIGHT = 2e-6   # GPU (float64 CG, float32 output) against the oracle with the same tolerances
GOLDEN = 1e-5  # against the reference's float64-tolerance goldens


def _setup(pre, **extra):
    data = load("projection_48x24x10")
    grid = grid_from(data)
    kw = dict(workloads.PLAIN_OPTIONS)
    kw.update(forcing=workloads.wind_forcing(grid), dt_bt=75.0, project_adv_vel=True,
              projection_preconditioner=pre, **extra)
    gpu = make_solver_global(grid, workloads.PLAIN_PHYSICS, 1800.0, **dict(kw, dtype="float32"))[0]
    oopts = {k: v for k, v in kw.items() if k in oparams.SUPPORTED}
    p32 = oparams.build_params(grid, workloads.PLAIN_PHYSICS, 1800.0, **dict(oopts, dtype="float32"))
    return data, grid, gpu, p32


def _state(grid, u, v):
    shape = (grid.nx, grid.ny, grid.nz)
    T = np.full(shape, workloads.PLAIN_PHYSICS.T_ref)
    S = np.full(shape, workloads.PLAIN_PHYSICS.S_ref)
    return dict(u=u, v=v, T=T, S=S, eta=np.zeros(shape[:2]))


@pytest.mark.parametrize("pre", ["none", "jacobi"])
def test_projection_matches_oracle_and_goldens(pre):
    data, grid, gpu, p32 = _setup(pre)
    got = gu.run_stage(gpu, 8, _state(grid, data["in_u"], data["in_v"]))
    ua, va = ostep.project_column_divergence(data["in_u"], data["in_v"], p32, 1800.0)
    errs = {"u": rel_l2(got["u"], ua), "v": rel_l2(got["v"], va)}
    assert max(errs.values()) < TIGHT, errs
    errs = {"u": rel_l2(got["u"], data[f"{pre}_u"]), "v": rel_l2(got["v"], data[f"{pre}_v"])}
    assert max(errs.values()) < GOLDEN, errs
    it = gpu.projection_stats()
    assert 1 <= it[0] <= p32.projection_niter, it
    # the column divergence is removed up to the solver tolerance
    before = np.linalg.norm(ostep.column_divergence(data["in_u"], data["in_v"], p32))
    after = np.linalg.norm(ostep.column_divergence(got["u"], got["v"], p32))
    assert after < 1e-4 * before, (after, before)


def test_projection_iteration_cap_matches_oracle():
    """projection_niter caps every solve (jax cg maxiter); three iterations do
    not converge, so each solve runs exactly three."""
    data, grid, gpu, p32 = _setup("none", projection_niter=3)
    got = gu.run_stage(gpu, 8, _state(grid, data["in_u"], data["in_v"]))
    ua, va = ostep.project_column_divergence(data["in_u"], data["in_v"], p32, 1800.0)
    errs = {"u": rel_l2(got["u"], ua), "v": rel_l2(got["v"], va)}
    assert max(errs.values()) < TIGHT, errs
    it = gpu.projection_stats()
    assert it[0] == 3 and it[3] == 2 and it[1] == 3 and it[2] == 3, it


def test_projection_without_refinements():
    data, grid, gpu, p32 = _setup("jacobi", projection_max_refinements=0, projection_niter=5)
    got = gu.run_stage(gpu, 8, _state(grid, data["in_u"], data["in_v"]))
    ua, va = ostep.project_column_divergence(data["in_u"], data["in_v"], p32, 1800.0)
    errs = {"u": rel_l2(got["u"], ua), "v": rel_l2(got["v"], va)}
    assert max(errs.values()) < TIGHT, errs
    assert gpu.projection_stats()[3] == 0


def test_projected_steps_match_reference_goldens():
    """The preset's projected step (reference, float64 tolerances) after 1 and 2 steps."""
    data = load("step_projected_48x24x10")
    grid, physics, dt, options, state = case_inputs(data)
    gpu, _ = gu.build_pair(grid, physics, dt, options)
    for n in (1, 2):
        got = gu.run_steps(gpu, state, n)
        want = {k: data[f"out{n}_{k}"] for k in gu.FIELDS}
        errs = gu.errors(got, want)
        assert max(errs.values()) < GOLDEN, (n, errs)


def test_projected_full_step_matches_oracle():
    """One projected step against the oracle with the float32 tolerances."""
    data = load("step_projected_48x24x10")
    grid, physics, dt, options, state = case_inputs(data)
    gpu = make_solver_global(grid, physics, dt, **dict(options, dtype="float32"))[0]
    oopts = {k: v for k, v in options.items() if k in oparams.SUPPORTED}
    p32 = oparams.build_params(grid, physics, dt, **dict(oopts, dtype="float32"))
    got = gu.run_stage(gpu, 3, state)
    want = ostep.step(gu.f32(state), p32)
    errs = gu.errors(got, want)
    assert max(errs.values()) < 1e-5, errs


def test_projection_is_deterministic_at_full_size():
    """720x360x50: the fixed-order reductions give the same bits on every run,
    the divergence drops, and the iteration counts stay within the cap."""
    import torch
    grid, physics, dt, kw, T, S = workloads.make_case("plain", 720, 360, 50, dtype="float32")
    step = make_solver_global(grid, physics, dt, **dict(kw, project_adv_vel=True))[0]
    rng = np.random.default_rng(5)
    wet = np.asarray(grid.wet_mask_3d)
    u = (0.2 * rng.standard_normal(wet.shape) * wet).astype(np.float32)
    v = (0.2 * rng.standard_normal(wet.shape) * wet).astype(np.float32)
    st = _state(grid, u, v)
    st["T"], st["S"] = T, S
    a = gu.run_stage(step, 8, st)
    it = step.projection_stats()
    b = gu.run_stage(step, 8, st)
    assert np.array_equal(a["u"], b["u"]) and np.array_equal(a["v"], b["v"])
    assert step.projection_stats() == it
    assert 1 <= it[0] <= 150 and 0 <= it[3] <= 2, it
    oopts = {k: v for k, v in kw.items() if k in oparams.SUPPORTED}
    p = oparams.build_params(grid, physics, dt, **dict(oopts, dtype="float32", project_adv_vel=True))
    before = np.linalg.norm(ostep.column_divergence(u.astype(np.float64), v.astype(np.float64), p))
    after = np.linalg.norm(ostep.column_divergence(a["u"], a["v"], p))
    assert after < 0.5 * before, (after, before)
    torch.cuda.synchronize()
