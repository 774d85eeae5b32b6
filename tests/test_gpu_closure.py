"""The learned vertical-mixing closure inside the step: its features and
plain-closure targets against the float64 oracle, the fused tensor-core
inference against the standalone one, the fallback to the plain closure, and
a stable run of the step with the closure on."""
import numpy as np
import pytest

from oracle import mlp as omlp
from oracle import params as oparams
from zhenmode_b200 import JaxStateG, make_solver_global, workloads

pytestmark = pytest.mark.gpu


def _case(nx=96, ny=48, nz=20):
    import torch
    grid, physics, dt, kw, T, S = workloads.make_case("plain", nx, ny, nz, dtype="float32")
    step, init, _ = make_solver_global(grid, physics, dt, **kw)
    oo = {k: v for k, v in kw.items() if k in oparams.SUPPORTED}
    oo["dtype"] = "float64"
    p = oparams.build_params(grid, physics, dt, **oo)
    st = init(T, S)
    rng = np.random.default_rng(2)
    wet3 = torch.as_tensor(np.asarray(grid.wet_mask_3d, np.float32), device="cuda")
    st = JaxStateG(st.u + 0.05 * torch.as_tensor(rng.standard_normal(st.u.shape), device="cuda",
                                                 dtype=torch.float32) * wet3,
                   st.v, st.T - 3.0 * ((torch.rand_like(st.T) < 0.02) & (wet3 > 0)).float(), st.S, st.eta,
                   st.ice)
    return grid, p, step, st


def test_features_match_oracle():
    grid, p, step, st = _case()
    X, T, M = (a.cpu().numpy() for a in step.closure_features(st))
    host = {k: getattr(st, k).cpu().numpy() for k in ("u", "v", "T", "S")}
    wX, wT, wM = omlp.closure_features(host, p)
    assert np.array_equal(M, wM)
    assert np.max(np.abs(X - wX)) < 1e-4 * max(1.0, np.max(np.abs(wX)))
    assert np.max(np.abs((T - wT) * wM)) < 1e-5
    assert np.any((wT > -3.0) & (wM > 0))   # some convecting interfaces in the case


def test_fused_inference_and_fallback():
    import torch
    from zhenmode_b200.closure import ClosureMLP
    grid, p, step, st = _case()
    net = ClosureMLP(seed=5)
    step.set_closure(net, bound=1e6)
    K = step.closure_kappa(st).cpu().numpy()
    X, T, M = step.closure_features(st)
    y = net.forward_bf16(X).cpu().numpy()
    want = np.clip(10.0 ** y.astype(np.float64), 1e-7, 1.0) * M.cpu().numpy()
    assert np.max(np.abs(K - want) / np.maximum(want, 1e-30) * (want > 0)) < 1e-3
    assert step.closure_stats() == (0, 0)
    # a bound below every feature: each wet column takes the plain closure
    step.set_closure(net, bound=1e-30)
    K = step.closure_kappa(st).cpu().numpy()
    Mn = M.cpu().numpy()
    plain = 10.0 ** T.cpu().numpy().astype(np.float64) * Mn
    assert np.max(np.abs(K - plain) / np.maximum(plain, 1e-30) * (Mn > 0)) < 1e-5
    assert step.closure_stats()[0] >= int((Mn.sum(1) > 0).sum())
    step.set_closure(None)


def test_step_with_closure_is_stable():
    """A few steps with an untrained network (kappa near 1e-6) stay finite and
    pass the monitor; the closure shows up in the launch count."""
    from zhenmode_b200.closure import ClosureMLP
    grid, p, step, st = _case()
    plain = step(st)
    step.set_closure(ClosureMLP(seed=1))
    out = st
    for _ in range(4):
        out = step(out)
    for k in ("u", "v", "T", "S", "eta"):
        assert bool(getattr(out, k).isfinite().all())
    assert float(out.u.abs().max()) < 10.0
    assert step.closure_stats()[1] == 0
    step.set_closure(None)
    again = step(st)
    assert all(bool((getattr(plain, k) == getattr(again, k)).all()) for k in ("u", "v", "T", "S", "eta"))


def test_trained_closure_tracks_the_plain_run():
    """Train the network on rows of the plain model itself (1 day, 180x90x50,
    cold surface patches that convect), then run one day from an unseen
    state: the daily-mean SST of the learned form stays within 0.05 K RMS of
    the plain run, and well inside what the same form gives without the
    network (a constant kappa_v, no convective mixing)."""
    import torch
    from zhenmode_b200.closure import ClosureMLP, collect, fit, init_params
    nx, ny, nz, nsteps = 180, 90, 50, 48
    grid, physics, dt, kw, T, S = workloads.make_case("plain", nx, ny, nz, dtype="float32")
    step, init, _ = make_solver_global(grid, physics, dt, **kw)
    wet3 = torch.as_tensor(np.asarray(grid.wet_mask_3d, np.float32), device="cuda")

    def patched(seed):
        st = init(T, S)
        g = torch.Generator(device="cpu").manual_seed(seed)
        patch = (torch.rand((nx, ny), generator=g) < 0.15).float().to("cuda")
        cool = torch.zeros_like(st.T)
        cool[:, :, :4] = 2.5 * patch[:, :, None]
        return JaxStateG(st.u, st.v, st.T - cool * wet3, st.S, st.eta, st.ice)

    def daily_sst(st):
        acc = torch.zeros((nx, ny), device="cuda")
        for _ in range(nsteps):
            st = step(st)
            acc += st.T[:, :, 0]
        return acc / nsteps

    X, Tt, M, _ = collect(step, patched(1), nsteps, every=2)
    net = ClosureMLP(seed=0)
    loss = fit(net, X, Tt, M, steps=3000, batch=8192, lr=1e-3)
    assert loss < 0.1, loss
    st0 = patched(2)
    ref = daily_sst(st0)
    step.set_closure(net)
    learned = daily_sst(st0)
    assert step.closure_stats() == (0, 0)
    plain_kv = init_params(0)
    plain_kv[:] = 0.0
    plain_kv[-64:] = np.log10(physics.kappa_v)
    step.set_closure(plain_kv)
    without = daily_sst(st0)
    step.set_closure(None)
    wet = torch.as_tensor(np.asarray(grid.wet_mask), device="cuda") > 0
    rmse = lambda a: float(torch.sqrt(((a - ref)[wet] ** 2).mean()))
    print(f"daily-mean SST RMSE vs plain: learned {rmse(learned):.4f} K, without the network {rmse(without):.4f} K")
    assert rmse(learned) <= 0.05
    assert rmse(without) > 4.0 * rmse(learned)
