"""The learned-closure MLP kernels against the float64 CPU oracle
(oracle/mlp.py): tensor-core BF16 inference, float32 gradients of the masked
mean-square loss, and Adam training."""
import numpy as np
import pytest

from oracle import mlp as omlp

pytestmark = pytest.mark.gpu

INFER_TOL = 5e-3     # BF16 operands; accumulation order and GELU rounding differ
GRAD_TOL = 1e-4      # float32 GPU gradients against float64


def _bf16(a):
    import torch
    return torch.as_tensor(np.asarray(a, dtype=np.float32)).to(torch.bfloat16).to(torch.float32).double().numpy()


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("ncol", [128, 1000])
def test_tensor_core_inference_matches_oracle(ncol):
    import torch
    from zhenmode_b200.closure import ClosureMLP, init_params
    p = init_params(seed=3, out_bias=0.5)
    p[:] += np.random.default_rng(4).standard_normal(p.size).astype(np.float32) * 0.01
    net = ClosureMLP(p)
    X = np.random.default_rng(5).standard_normal((ncol, 256)).astype(np.float32)
    X[:, 252:] = 0.0
    got = net.forward_bf16(torch.as_tensor(X, device="cuda")).cpu().numpy()
    net.check_error()
    want = omlp.forward_bf16(p, X, _bf16)
    assert _rel(got, want) < INFER_TOL, _rel(got, want)
    # a second call on the same object gives the same bits
    again = net.forward_bf16(torch.as_tensor(X, device="cuda")).cpu().numpy()
    assert np.array_equal(got, again)


def test_gradients_match_oracle():
    import torch
    from zhenmode_b200.closure import ClosureMLP, init_params
    rng = np.random.default_rng(7)
    p = init_params(seed=8, out_bias=0.0)
    B = 96
    X = rng.standard_normal((B, 256)).astype(np.float32)
    T = rng.standard_normal((B, 64)).astype(np.float32)
    M = (rng.random((B, 64)) < 0.7).astype(np.float32)
    net = ClosureMLP(p)
    loss, g = net.grad(*(torch.as_tensor(a, device="cuda") for a in (X, T, M)))
    want_loss, want_g = omlp.loss_and_grad(p, X, T, M)
    assert abs(loss - want_loss) <= GRAD_TOL * want_loss
    g = g.cpu().numpy()
    for name in omlp.OFF:
        sl = slice(omlp.OFF[name], omlp.OFF[name] + int(np.prod(omlp.SHAPES[name])))
        assert _rel(g[sl], want_g[sl]) < GRAD_TOL, (name, _rel(g[sl], want_g[sl]))


def test_training_reduces_loss():
    """Adam on a smooth synthetic map: the loss falls by more than 10x."""
    import torch
    from zhenmode_b200.closure import ClosureMLP
    rng = np.random.default_rng(11)
    B = 2048
    X = rng.standard_normal((B, 256)).astype(np.float32) * 0.5
    A = rng.standard_normal((256, 64)).astype(np.float32) / 16.0
    T = np.tanh(X @ A).astype(np.float32)
    M = np.ones_like(T)
    net = ClosureMLP(seed=1)
    net.params[-64:] = 0.0
    Xd, Td, Md = (torch.as_tensor(a, device="cuda") for a in (X, T, M))
    first = net.grad(Xd, Td, Md)[0]
    for _ in range(300):
        net.train_step(Xd, Td, Md, lr=2e-3)
    last = net.grad(Xd, Td, Md)[0]
    assert last < first / 10.0, (first, last)
