"""The learned-preconditioner oracle (FP64 numpy) against finite differences:
pins the analytic gradients that the GPU kernels are compared with."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
from oracle import mlp as O  # noqa: E402


def _problem(n=7, F=6, H=5, D=6, K=2, seed=0):
    g = np.random.default_rng(seed)
    X = g.normal(size=(n, F))
    params = [g.normal(size=(H, F)) * 0.5, g.normal(size=H) * 0.1, g.normal(size=(H, H)) * 0.5, g.normal(size=H) * 0.1,
              g.normal(size=(D * K + 1, H)) * 0.3, g.normal(size=D * K + 1) * 0.1]
    U = g.normal(size=(n, 9, D))
    Tt = g.normal(size=(n, 9, D))
    C = np.einsum("nsd,nse->nde", U, U)
    Gr = np.einsum("nsd,nse->nde", U, Tt)
    G = 0.5 * (Gr + np.transpose(Gr, (0, 2, 1)))
    T = np.einsum("nsd,nsd->n", Tt, Tt)
    return X, params, C, G, T, D, K


def test_loss_is_the_squared_error():
    # J_b = Sum_s || (L L^T + d I) u_s - t_s ||^2 for explicit samples
    g = np.random.default_rng(1)
    D, K, S = 6, 2, 11
    L = g.normal(size=(1, D, K))
    d = np.array([0.37])
    u = g.normal(size=(S, D))
    t = g.normal(size=(S, D))
    C = (u.T @ u)[None]
    Gr = u.T @ t
    G = (0.5 * (Gr + Gr.T))[None]
    T = np.array([np.sum(t * t)])
    J, _, _ = O.block_loss(L, d, C, G, T)
    P = L[0] @ L[0].T + d[0] * np.eye(D)
    want = sum(np.sum((P @ u[s] - t[s]) ** 2) for s in range(S))
    assert abs(J[0] - want) <= 1e-10 * want


def test_gradients_match_finite_differences():
    X, params, C, G, T, D, K = _problem()
    loss, grads = O.loss_and_grads(X, params, C, G, T, D, K)
    h = 1e-6
    for pi, (p, gp) in enumerate(zip(params, grads)):
        flat = p.reshape(-1)
        for k in range(0, flat.size, max(1, flat.size // 7)):
            old = flat[k]
            flat[k] = old + h
            lp, _ = O.loss_and_grads(X, params, C, G, T, D, K)
            flat[k] = old - h
            lm, _ = O.loss_and_grads(X, params, C, G, T, D, K)
            flat[k] = old
            fd = (lp - lm) / (2 * h)
            assert abs(fd - gp.reshape(-1)[k]) <= 1e-6 * max(1.0, abs(fd)), (pi, k, fd, gp.reshape(-1)[k])
