"""``jax.scipy.sparse.linalg`` stand-in.  Test infrastructure only.

``cg`` restates the preconditioned conjugate-gradient loop of
jax.scipy.sparse.linalg.cg (jax 0.11.2, pinned by the reference's
requirements.txt; the published ``_cg_solve``): x0 = 0, r0 = b - A x0,
p0 = z0 = M r0, gamma0 = <r0, z0>; repeat while the squared residual norm
(gamma when M is the identity, else <r, r>) exceeds max(tol^2 <b, b>, atol^2)
and fewer than maxiter iterations ran: alpha = gamma / <p, A p>,
x += alpha p, r -= alpha A p, z = M r, gamma' = <r, z>, beta = gamma' / gamma,
p = z + beta p.  Returns (x, None) like jax.
"""
import numpy as np


def cg(A, b, x0=None, *, tol=1e-5, atol=0.0, maxiter=None, M=None):
    b = np.asarray(b, dtype=np.float64)
    if maxiter is None:
        maxiter = 10 * b.size
    identity = M is None
    precond = (lambda r: r) if identity else M
    x = np.zeros_like(b) if x0 is None else np.asarray(x0, dtype=np.float64)
    bs = float(np.vdot(b, b))
    atol2 = max(tol * tol * bs, atol * atol)
    r = b - np.asarray(A(x))
    z = np.asarray(precond(r))
    p = z
    gamma = float(np.vdot(r, z))
    k = 0
    while True:
        rs = gamma if identity else float(np.vdot(r, r))
        if not (rs > atol2 and k < maxiter):
            break
        Ap = np.asarray(A(p))
        alpha = gamma / float(np.vdot(p, Ap))
        x = x + alpha * p
        r = r - alpha * Ap
        z = np.asarray(precond(r))
        gamma_new = float(np.vdot(r, z))
        beta = gamma_new / gamma
        p = z + beta * p
        gamma = gamma_new
        k += 1
    return x, None
