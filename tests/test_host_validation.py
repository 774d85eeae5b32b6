"""Host-side behaviour of the drop-in factory that needs no GPU: invalid
configurations raise ValueError before anything is built (as the reference
factory does, src/zhenmode/model/solver/factory.py:166-395), and options the
B200 path lacks raise UnsupportedOption (a ValueError subclass)."""
import dataclasses

import numpy as np
import pytest

from zhenmode_b200 import UnsupportedOption, make_solver_global, workloads


@pytest.fixture(scope="module")
def case():
    return workloads.make_case("plain", 24, 12, 6, dtype="float32")


def _call(case, **over):
    grid, physics, dt, kw, _, _ = case
    kw = dict(kw)
    kw.update(over)
    return make_solver_global(grid, physics, dt, **kw)


@pytest.mark.parametrize("over", [dict(dt_bt=0.0), dict(dt_bt=float("nan")), dict(polar_cap_rows=-1),
                                  dict(polar_cap_rows=4, polar_cap_taper=3), dict(dtype="float16"),
                                  dict(nu_nsub=0), dict(lambda_bulk=-1.0), dict(process_time_scheme="bogus"),
                                  dict(column_geometry="bogus"), dict(vertical_diffusion="crank"),
                                  dict(projection_max_refinements=3)])
def test_invalid_configuration_raises_value_error(case, over):
    with pytest.raises(ValueError):
        _call(case, **over)


def test_invalid_dt_and_physics(case):
    grid, physics, dt, kw, _, _ = case
    with pytest.raises(ValueError):
        make_solver_global(grid, physics, -1.0, **kw)
    with pytest.raises(ValueError):
        make_solver_global(grid, dataclasses.replace(physics, nu_h=-1.0), dt, **kw)


def test_invalid_grid(case):
    grid, physics, dt, kw, _, _ = case
    bad = dataclasses.replace(grid, z=np.asarray(grid.z)[::-1].copy())
    with pytest.raises(ValueError):
        make_solver_global(bad, physics, dt, **kw)


@pytest.mark.parametrize("over", [dict(mode_split=False), dict(dtype="float64"),
                                  dict(dynamic_ice=True),
                                  dict(mixed_layer_depth_m=50.0)])
def test_unsupported_options(case, over):
    with pytest.raises(UnsupportedOption):
        _call(case, **over)


@pytest.mark.parametrize("over", [dict(projection_niter=0), dict(projection_niter=True), dict(projection_niter=2.5),
                                  dict(projection_rtol=0.0), dict(projection_rtol=float("nan")),
                                  dict(projection_preconditioner="ilu"), dict(projection_max_refinements=3),
                                  dict(projection_max_refinements=-1)])
def test_invalid_projection_options(case, over):
    """factory.py:377-384: the projection options are checked whether or not it is on."""
    with pytest.raises(ValueError):
        _call(case, **over)


def test_projection_niter_environment(case, monkeypatch):
    """factory.py:368-376: OCEAN_PAV_NITER stands in for projection_niter=None."""
    monkeypatch.setenv("OCEAN_PAV_NITER", "many")
    with pytest.raises(ValueError, match="environment"):
        _call(case, project_adv_vel=True)
    monkeypatch.setenv("OCEAN_PAV_NITER", "0")
    with pytest.raises(ValueError, match="positive"):
        _call(case, project_adv_vel=True)


def test_unknown_scheme_keyword(case):
    with pytest.raises(TypeError):
        _call(case, not_an_option=1)
    with pytest.raises(ValueError):
        _call(case, vertical_tracer_scheme="bogus")


def test_more_than_64_levels_is_unsupported():
    """The 3-D wet mask is one 64-bit word per column: nz <= 64."""
    grid, physics, dt, kw, _, _ = workloads.make_case("plain", 24, 12, 65, dtype="float32")
    with pytest.raises(UnsupportedOption):
        make_solver_global(grid, physics, dt, **kw)
