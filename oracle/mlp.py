"""ORACLE (test infrastructure only): float64 NumPy restatement of the
learned-closure MLP (256 -> 256 -> 256 -> 64, exact GELU) with its
masked mean-square loss and gradients, and a BF16-rounding emulation of the
tensor-core inference.  The MLP is new (no reference counterpart); this file
is the CPU oracle its GPU forward and backward kernels are checked against.

Only ``tests/`` import this module.
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf

OFF = dict(W1=0, b1=65536, W2=65792, b2=131328, W3=131584, b3=147968)
SHAPES = dict(W1=(256, 256), b1=(256,), W2=(256, 256), b2=(256,), W3=(64, 256), b3=(64,))


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return {k: p[OFF[k]:OFF[k] + int(np.prod(s))].reshape(s) for k, s in SHAPES.items()}


def gelu(x):
    return 0.5 * x * (1.0 + erf(x / np.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + erf(x / np.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / np.sqrt(2.0 * np.pi)


def forward(p, X):
    w = unpack(p)
    Z1 = X @ w["W1"].T + w["b1"]
    H1 = gelu(Z1)
    Z2 = H1 @ w["W2"].T + w["b2"]
    H2 = gelu(Z2)
    return H2 @ w["W3"].T + w["b3"], (Z1, H1, Z2, H2)


def loss_and_grad(p, X, T, M):
    """Masked mean-square loss sum(M (Y - T)^2) / sum(M) and its gradient,
    packed like the parameters."""
    X = np.asarray(X, dtype=np.float64)
    w = unpack(p)
    Y, (Z1, H1, Z2, H2) = forward(p, X)
    cnt = float(np.sum(M))
    E = (Y - T) * M
    loss = float(np.sum(E * E) / cnt)
    dY = 2.0 * E / cnt
    g = {}
    g["W3"] = dY.T @ H2
    g["b3"] = dY.sum(0)
    dZ2 = (dY @ w["W3"]) * gelu_grad(Z2)
    g["W2"] = dZ2.T @ H1
    g["b2"] = dZ2.sum(0)
    dZ1 = (dZ2 @ w["W2"]) * gelu_grad(Z1)
    g["W1"] = dZ1.T @ X
    g["b1"] = dZ1.sum(0)
    out = np.zeros(len(np.asarray(p)), dtype=np.float64)
    for k in OFF:
        out[OFF[k]:OFF[k] + g[k].size] = g[k].ravel()
    return loss, out


def forward_bf16(p, X, round_bf16):
    """Inference with BF16 operands as the tensor cores see them: inputs,
    weights and the two hidden activations rounded by ``round_bf16``; float64
    accumulation and float32-exact biases."""
    w = unpack(p)
    r = round_bf16
    H = r(np.asarray(X, dtype=np.float64))
    H = r(gelu(H @ r(w["W1"]).T + w["b1"]))
    H = r(gelu(H @ r(w["W2"]).T + w["b2"]))
    return H @ r(w["W3"]).T + w["b3"]


def closure_features(state, p):
    """Float64 training rows of a state (the closure's features and the
    plain closure's log10 diffusivity per interface, physics/vertical.py:40-82),
    rows j-major with i fastest, as the GPU kernel writes them."""
    T = np.asarray(state["T"], np.float64) - p.T_ref
    S = np.asarray(state["S"], np.float64) - p.S_ref
    u = np.asarray(state["u"], np.float64)
    v = np.asarray(state["v"], np.float64)
    wm = np.asarray(p.wet_mask_z, np.float64)
    nx, ny, nz = T.shape
    X = np.zeros((nx, ny, 256))
    X[..., 0:nz] = T * 0.1 * wm
    X[..., 50:50 + nz] = S * wm
    X[..., 100:100 + nz] = u * 2.0 * wm
    X[..., 150:150 + nz] = v * 2.0 * wm
    wif = wm[..., :-1] * wm[..., 1:]
    dz = np.asarray(p.dz_3d, np.float64).reshape(-1)
    n2 = 9.81 * (-2.0e-4 * (T[..., 1:] - T[..., :-1]) + 7.6e-4 * (S[..., 1:] - S[..., :-1])) / dz
    X[..., 200:200 + nz - 1] = np.arcsinh(n2 * 1e8) * 0.25 * wif
    X[..., 250] = np.hypot(p.tau_x_2d, p.tau_y_2d) * 10.0
    X[..., 251] = p.Q_heat_2d * 0.01
    unstable = (7.6e-4 * (S[..., :-1] - S[..., 1:]) > 2.0e-4 * (T[..., :-1] - T[..., 1:])) & (wif > 0.5)
    col = np.any(unstable, axis=-1, keepdims=True)
    gate = unstable if p.localize_conv else np.broadcast_to(col, unstable.shape)
    kap = p.kappa_v + p.coastal_kappa_v_2d[..., None] + (p.kappa_conv if p.kappa_conv > 0 else 0.0) * gate
    Tt = np.zeros((nx, ny, 64))
    M = np.zeros((nx, ny, 64))
    Tt[..., :nz - 1] = np.where(wif > 0.5, np.log10(np.where(wif > 0.5, kap, 1.0)), 0.0)
    M[..., :nz - 1] = wif
    rows = lambda a: np.transpose(a, (1, 0, 2)).reshape(nx * ny, -1)
    return rows(X), rows(Tt), rows(M)
