"""CPU oracle (test infrastructure only) of the learned band preconditioner's
training and application kernels (libpscuda ps_lbp_* / ps_mlp_*): FP64 numpy,
same formulas.  There is no reference counterpart (the reference's CG has no
learned preconditioner); the oracle is pinned by finite differences
(tests/test_learned_oracle.py).

Shapes: features X [n, F]; W1 [H, F], b1 [H]; W2 [H, H], b2 [H]; W3 [O, H], b3 [O];
O = D * K + 1: L = out[:, :D*K].reshape(n, D, K), q = out[:, -1], d = 0.5 tanh(q);
moments C, G [n, D, D] (symmetric), T [n].
"""
import numpy as np


def forward(X, params):
    W1, b1, W2, b2, W3, b3 = params
    h1 = np.maximum(X @ W1.T + b1, 0.0)
    h2 = np.maximum(h1 @ W2.T + b2, 0.0)
    out = h2 @ W3.T + b3
    return h1, h2, out


def block_loss(L, d, C, G, T):
    """J_b = || (L L^T + d I) u - t ||^2 over the pairs, from the moments:
    tr(B A) + 2 d tr(B) + d^2 tr(C) - 2 tr(L^T G L) - 2 d tr(G) + T  (A = L^T L, B = L^T C L);
    dJ/dL = 2 (C L A + L B + 2 d C L - 2 G L),  dJ/dd = 2 (tr(B) + d tr(C) - tr(G))."""
    A = np.einsum("nda,ndc->nac", L, L)
    CL = np.einsum("nde,nea->nda", C, L)
    GL = np.einsum("nde,nea->nda", G, L)
    Bm = np.einsum("nda,ndc->nac", L, CL)
    trB = np.einsum("naa->n", Bm)
    trC = np.einsum("naa->n", C)
    trG = np.einsum("naa->n", G)
    J = (np.einsum("nac,nca->n", Bm, A) + 2 * d * trB + d * d * trC - 2.0 * np.einsum("nda,nda->n", L, GL)
         - 2 * d * trG + T)
    dL = 2.0 * (np.einsum("nda,nac->ndc", CL, A) + np.einsum("nda,nac->ndc", L, Bm) + 2 * d[:, None, None] * CL
                - 2.0 * GL)
    dd = 2.0 * (trB + d * trC - trG)
    return J, dL, dd


def loss_and_grads(X, params, C, G, T, D, K):
    """Normalised loss Sum_b J_b / Sum_b T_b and its gradients w.r.t. the six parameters."""
    W1, b1, W2, b2, W3, b3 = params
    h1, h2, out = forward(X, params)
    n = X.shape[0]
    L = out[:, :D * K].reshape(n, D, K)
    th = np.tanh(out[:, D * K])
    J, dL, dd = block_loss(L, 0.5 * th, C, G, T)
    s = 1.0 / np.sum(T)
    d3 = np.concatenate([dL.reshape(n, -1), (dd * 0.5 * (1 - th * th))[:, None]], axis=1) * s
    gW3, gb3 = d3.T @ h2, d3.sum(0)
    d2 = (d3 @ W3) * (h2 > 0)
    gW2, gb2 = d2.T @ h1, d2.sum(0)
    d1 = (d2 @ W2) * (h1 > 0)
    gW1, gb1 = d1.T @ X, d1.sum(0)
    return float(np.sum(J) * s), [gW1, gb1, gW2, gb2, gW3, gb3]


def moments(blocks, r, e, w, sigma, band_l):
    """Per-block C, G, T from pairs r, e [B, 3, nalm] complex (see ps_lbp_moments).
    blocks: list of (alm index of the first l, number of valid l)."""
    D = 3 * band_l
    nb = len(blocks)
    C = np.zeros((nb, D, D))
    G = np.zeros((nb, D, D))
    T = np.zeros(nb)
    S = np.einsum("ffi->fi", sigma)
    Sr = np.einsum("fgi,ngi->nfi", sigma, r)
    for b, (i0, nl) in enumerate(blocks):
        for n in range(r.shape[0]):
            u = np.zeros((2, D))
            t = np.zeros((2, D))
            for f in range(3):
                sl = slice(i0, i0 + nl)
                sq = np.sqrt(np.maximum(S[f, sl], 0.0))
                isq = np.where(S[f, sl] > 0, 1.0 / np.sqrt(np.where(S[f, sl] > 0, S[f, sl], 1.0)), 0.0)
                u[0, f * band_l:f * band_l + nl] = sq * r[n, f, sl].real
                u[1, f * band_l:f * band_l + nl] = sq * r[n, f, sl].imag
                t[0, f * band_l:f * band_l + nl] = isq * (e[n, f, sl].real - Sr[n, f, sl].real)
                t[1, f * band_l:f * band_l + nl] = isq * (e[n, f, sl].imag - Sr[n, f, sl].imag)
            C[b] += w[n] * (np.outer(u[0], u[0]) + np.outer(u[1], u[1]))
            ut = np.outer(u[0], t[0]) + np.outer(u[1], t[1])
            G[b] += w[n] * 0.5 * (ut + ut.T)
            T[b] += w[n] * np.sum(t ** 2)
    return C, G, T


def apply(blocks, L, sigma, r, band_l):
    """M r = Sigma r + S^1/2 (L L^T + d I) S^1/2 r on every block (see ps_lbp_apply);
    L [nb, D*K + 1] network outputs."""
    z = np.einsum("fgi,ngi->nfi", sigma, r)
    S = np.einsum("ffi->fi", sigma)
    D = 3 * band_l
    for b, (i0, nl) in enumerate(blocks):
        for n in range(r.shape[0]):
            u = np.zeros(D, dtype=complex)
            sq = np.zeros(D)
            for f in range(3):
                sl = slice(i0, i0 + nl)
                sq[f * band_l:f * band_l + nl] = np.sqrt(np.maximum(S[f, sl], 0.0))
                u[f * band_l:f * band_l + nl] = r[n, f, sl]
            Lb = L[b][:-1].reshape(D, -1)
            c = sq * (Lb @ (Lb.T @ (sq * u)) + 0.5 * np.tanh(L[b][-1]) * (sq * u))
            for f in range(3):
                z[n, f, i0:i0 + nl] += c[f * band_l:f * band_l + nl]
    return z
