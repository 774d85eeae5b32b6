"""Learned vertical-mixing closure: the per-column MLP and its training.

The network stands in for the plain closure of the reference
(``_effective_kappa_v`` and ``_convective_mask``, physics/vertical.py:40-82):
kappa_v + coastal band + kappa_conv on statically unstable interfaces.  It
maps 252 column features (T, S, u, v over 50 levels, N^2 on a signed log
scale over 49 interfaces, wind stress magnitude, heat flux; 4 zero pads) to 64 outputs, of which
outputs 0..nz-2 are log10 of the diffusivity at interfaces 0..nz-2 and the
rest are unused.

All arithmetic runs in ``libzm_b200.so``: inference on the tensor cores in
BF16 with float32 accumulation (``zm_mlp_forward_bf16``), training in float32
(``zm_mlp_grad``, ``zm_mlp_train_step``).  PyTorch only holds the device
arrays.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native

N_IN, N_OUT = 256, 64
N_PARAMS = 148032
_OFF = dict(W1=0, b1=65536, W2=65792, b2=131328, W3=131584, b3=147968)
_SHAPES = dict(W1=(256, 256), b1=(256,), W2=(256, 256), b2=(256,), W3=(64, 256), b3=(64,))


def init_params(seed=0, out_bias=-6.0):
    """Seeded float32 parameters (scaled normal weights, zero hidden biases,
    output biases at ``out_bias``) as a flat NumPy array."""
    rng = np.random.default_rng(seed)
    p = np.zeros(N_PARAMS, dtype=np.float32)
    for name, fan_in in (("W1", 256), ("W2", 256), ("W3", 256)):
        n = int(np.prod(_SHAPES[name]))
        p[_OFF[name]:_OFF[name] + n] = (rng.standard_normal(n) * np.sqrt(1.0 / fan_in)).astype(np.float32)
    p[_OFF["b3"]:_OFF["b3"] + 64] = out_bias
    return p


def unpack(params):
    """dict of the parameter blocks (views) of a flat array or tensor."""
    return {k: params[_OFF[k]:_OFF[k] + int(np.prod(s))].reshape(s) for k, s in _SHAPES.items()}


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream(t):
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)


def _check(rc, what):
    if rc != _native.ZM_OK:
        raise RuntimeError(f"{what} failed with status {rc}")


class ClosureMLP:
    """The closure network on one GPU: float32 master parameters, BF16 copies
    for inference, Adam state for training."""

    def __init__(self, params=None, seed=0, device="cuda"):
        import torch
        self.lib = _native.load()
        p = init_params(seed) if params is None else np.asarray(params, dtype=np.float32)
        if p.shape != (N_PARAMS,):
            raise ValueError(f"expected {N_PARAMS} parameters, got {p.shape}")
        self.params = torch.as_tensor(p, device=device).clone()
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.step_count = 0
        self._tr = None
        self._tr_batch = 0
        self.err = torch.zeros(1, dtype=torch.int32, device=device)
        self.pack()

    # ---- inference
    def pack(self):
        """Refresh the BF16 weight copies from the float32 parameters."""
        import torch
        dev = self.params.device
        self.W1 = torch.empty((256, 256), dtype=torch.bfloat16, device=dev)
        self.W2 = torch.empty((256, 256), dtype=torch.bfloat16, device=dev)
        self.W3 = torch.empty((64, 256), dtype=torch.bfloat16, device=dev)
        _check(self.lib.zm_mlp_pack_bf16(_stream(self.params), _ptr(self.params), _ptr(self.W1), _ptr(self.W2),
                                         _ptr(self.W3)), "zm_mlp_pack_bf16")
        blocks = unpack(self.params)
        self.b1, self.b2, self.b3 = (blocks[k].contiguous() for k in ("b1", "b2", "b3"))

    def forward_bf16(self, X):
        """Tensor-core inference: X [n][256] (any float dtype, CUDA) -> [n][64] float32."""
        import torch
        Xb = X.to(torch.bfloat16).contiguous()
        if Xb.dim() != 2 or Xb.shape[1] != N_IN:
            raise ValueError("X must be [n][256]")
        Y = torch.empty((Xb.shape[0], N_OUT), dtype=torch.float32, device=Xb.device)
        _check(self.lib.zm_mlp_forward_bf16(_stream(Xb), int(Xb.shape[0]), _ptr(Xb), _ptr(self.W1), _ptr(self.b1),
                                            _ptr(self.W2), _ptr(self.b2), _ptr(self.W3), _ptr(self.b3), _ptr(Y),
                                            _ptr(self.err)), "zm_mlp_forward_bf16")
        return Y

    def check_error(self):
        if int(self.err.item()) != 0:
            raise RuntimeError("a tensor-core wait of the MLP ran out of polls")

    # ---- training
    def _trainer(self, batch):
        if self._tr is None or batch > self._tr_batch:
            if self._tr is not None:
                self.lib.zm_mlp_trainer_destroy(self._tr)
            h = ctypes.c_void_p()
            _check(self.lib.zm_mlp_trainer_create(int(batch), ctypes.byref(h)), "zm_mlp_trainer_create")
            self._tr, self._tr_batch = h, int(batch)
        return self._tr

    @staticmethod
    def _batch_args(X, T, M):
        import torch
        X, T, M = (a.to(torch.float32).contiguous() for a in (X, T, M))
        if X.shape[1] != N_IN or T.shape != (X.shape[0], N_OUT) or M.shape != T.shape:
            raise ValueError("X [B][256], T and M [B][64]")
        count = float(M.sum().item())
        if count <= 0:
            raise ValueError("the mask selects no output")
        return X, T, M, count

    def grad(self, X, T, M):
        """(loss, gradient) of the masked mean-square error on one batch (float32)."""
        import torch
        X, T, M, count = self._batch_args(X, T, M)
        g = torch.empty_like(self.params)
        loss = ctypes.c_double()
        _check(self.lib.zm_mlp_grad(self._trainer(X.shape[0]), _stream(X), int(X.shape[0]), _ptr(X), _ptr(T), _ptr(M),
                                    count, _ptr(self.params), _ptr(g), ctypes.byref(loss)), "zm_mlp_grad")
        return loss.value, g

    def train_step(self, X, T, M, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8, want_loss=False):
        """One Adam step on one batch; returns the batch loss when asked (synchronizes)."""
        X, T, M, count = self._batch_args(X, T, M)
        self.step_count += 1
        loss = ctypes.c_double()
        _check(self.lib.zm_mlp_train_step(self._trainer(X.shape[0]), _stream(X), int(X.shape[0]), _ptr(X), _ptr(T),
                                          _ptr(M), count, _ptr(self.params), _ptr(self.m), _ptr(self.v),
                                          int(self.step_count), float(lr), float(beta1), float(beta2), float(eps),
                                          ctypes.byref(loss) if want_loss else None), "zm_mlp_train_step")
        return loss.value if want_loss else None

    def __del__(self):
        tr = getattr(self, "_tr", None)
        if tr is not None:
            self.lib.zm_mlp_trainer_destroy(tr)
            self._tr = None


def collect(step, state, nsteps, every=1, max_rows=2_000_000, seed=0):
    """Run ``step`` (the plain closure) ``nsteps`` times from ``state`` and take
    the training rows of the wet columns every ``every`` steps; keep at most
    ``max_rows`` of them, spread evenly over the snapshots (seeded
    subsample).  Returns (X, T, M, final state)."""
    import torch
    g = torch.Generator(device="cpu").manual_seed(seed)
    per_snapshot = -(-max_rows // max(1, nsteps // every))
    parts = []
    for n in range(nsteps):
        state = step(state)
        if (n + 1) % every == 0:
            X, T, M = step.closure_features(state)
            keep = torch.nonzero(M.sum(1) > 0).squeeze(1)
            if keep.numel() > per_snapshot:
                keep = keep[torch.randperm(keep.numel(), generator=g)[:per_snapshot].to(keep.device)]
            parts.append((X[keep], T[keep], M[keep]))
    X = torch.cat([p[0] for p in parts])
    T = torch.cat([p[1] for p in parts])
    M = torch.cat([p[2] for p in parts])
    if X.shape[0] > max_rows:
        idx = torch.randperm(X.shape[0], generator=g)[:max_rows].to(X.device)
        X, T, M = X[idx], T[idx], M[idx]
    return X, T, M, state


def fit(net, X, T, M, steps=2000, batch=8192, lr=1e-3, seed=0):
    """Adam on random batches of the rows (the native float32 training
    kernels); returns the masked mean-square loss on all rows afterwards."""
    import torch
    g = torch.Generator(device="cpu").manual_seed(seed)
    n = X.shape[0]
    batch = min(batch, n)
    for _ in range(steps):
        idx = torch.randint(0, n, (batch,), generator=g).to(X.device)
        net.train_step(X[idx], T[idx], M[idx], lr=lr)
    net.pack()
    losses = []
    for a in range(0, n, 65536):
        sl = slice(a, min(n, a + 65536))
        losses.append(net.grad(X[sl], T[sl], M[sl])[0] * float(M[sl].sum().item()))
    return sum(losses) / float(M.sum().item())


def mixed_layer_depth(T, S, z, wet3, ref_depth=10.0, density_delta=0.03):
    """Density-threshold mixed-layer depth in metres, positive down, of every
    column (diagnostics/mixed_layer.py:39-74, linear density of :14-35):
    the depth of the first level at or below ``ref_depth`` whose density
    exceeds the density at the level nearest ``ref_depth`` by
    ``density_delta``; the deepest wet level where none does; NaN on land.
    Levels below the seafloor (``wet3`` == 0) are the missing profile levels
    of the reference.  Host NumPy over all columns at once; T, S and wet3 are
    (nx, ny, nz) arrays, z the (nz,) node depths (negative down)."""
    T = np.asarray(T, dtype=np.float64)
    S = np.asarray(S, dtype=np.float64)
    wet = np.asarray(wet3) > 0.5
    depth = -np.asarray(z, dtype=np.float64)
    rho = 1025.0 * (1.0 - 2.0e-4 * (T - 15.0) + 7.6e-4 * (S - 35.0))
    ref_k = int(np.argmin(np.abs(depth - ref_depth)))
    delta = rho - rho[..., ref_k:ref_k + 1]
    hit = wet & (depth >= ref_depth)[None, None, :] & (delta >= density_delta)
    first = np.argmax(hit, axis=-1)
    nz = T.shape[-1]
    deepest = nz - 1 - np.argmax(wet[..., ::-1], axis=-1)
    k = np.where(hit.any(axis=-1), first, deepest)
    mld = depth[k]
    # the reference needs the level nearest ref_depth to be valid for any delta
    ok = wet.any(axis=-1) & wet[..., ref_k]
    return np.where(ok, mld, np.where(wet.any(axis=-1), depth[deepest], np.nan))


def compare_with_plain(step, net, state, days, steps_per_day, grid):
    """Run ``days`` simulated days from ``state`` with the plain closure and
    with the network ``net`` (the plain closure judges the network), and
    return per-day RMSEs over the wet columns of the daily-mean SST, SSS and
    mixed-layer depth (from the daily-mean T and S) of the learned run
    against the plain run, with the fallback-column count of the last step."""
    import torch
    wet2 = np.asarray(grid.wet_mask) > 0.5
    wet3 = np.asarray(grid.wet_mask_3d)
    z = np.asarray(grid.z)

    def daily_means(closure):
        step.set_closure(closure)
        st, out = state, []
        for _ in range(days):
            accT = torch.zeros_like(state.T)
            accS = torch.zeros_like(state.S)
            for _ in range(steps_per_day):
                st = step(st)
                accT += st.T
                accS += st.S
            out.append((accT / steps_per_day, accS / steps_per_day))
        fallback = step.closure_stats()[0] if closure is not None else 0
        step.set_closure(None)
        return out, fallback

    plain, _ = daily_means(None)
    learned, fallback = daily_means(net)
    rmse = lambda a, b: float(np.sqrt(np.nanmean(((a - b)[wet2]) ** 2)))  # noqa: E731
    res = {"sst_rmse_K": [], "sss_rmse_psu": [], "mld_rmse_m": [], "mld_mean_m": []}
    for (tp, sp), (tl, sl) in zip(plain, learned):
        tp, sp, tl, sl = (a.cpu().numpy() for a in (tp, sp, tl, sl))
        res["sst_rmse_K"].append(rmse(tl[..., 0], tp[..., 0]))
        res["sss_rmse_psu"].append(rmse(sl[..., 0], sp[..., 0]))
        mp = mixed_layer_depth(tp, sp, z, wet3)
        ml = mixed_layer_depth(tl, sl, z, wet3)
        res["mld_rmse_m"].append(rmse(ml, mp))
        res["mld_mean_m"].append(float(np.nanmean(mp[wet2])))
    res["fallback_columns_last_step"] = int(fallback)
    return res
