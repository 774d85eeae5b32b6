"""The on-device seasonal forcing blend (inputs/forcing/seasonal.py:86-103):
a step after the device blend equals a step given the oracle-blended fields."""
import numpy as np
import pytest

from oracle import seasonal
from zhenmode_b200 import make_solver_global, workloads

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("day", [14.5, 28.7, 31.2])
def test_seasonal_blend_drives_the_step(day):
    import torch
    grid, physics, dt, kw, T, S = workloads.make_case("plain", 48, 24, 10, dtype="float32")
    step, init, _ = make_solver_global(grid, physics, dt, **kw)
    st = init(T, S)
    rng = np.random.default_rng(3)
    lat = np.radians(np.asarray(grid.lat))
    base = 0.1 * np.sin(2 * lat) * np.cos(lat)
    taux = np.stack([np.broadcast_to(base * (1 + 0.3 * np.sin(2 * np.pi * (m + 0.5) / 12)), (48, 24))
                     for m in range(12)]).astype(np.float32)
    q = (100.0 * rng.standard_normal((12, 48, 24))).astype(np.float32)
    step.set_forcing_seasonal(tau_x=taux, q_heat=q, day=day)
    a = step(st)
    step.set_forcing(tau_x=seasonal.blend(taux, day).astype(np.float32), q_heat=seasonal.blend(q, day).astype(np.float32))
    b = step(st)
    for k in ("u", "v", "T", "S", "eta"):
        x, y = getattr(a, k).cpu().numpy(), getattr(b, k).cpu().numpy()
        assert np.linalg.norm(x - y) <= 1e-6 * max(np.linalg.norm(y), 1e-30), k
