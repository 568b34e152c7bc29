"""Harmonic-space vector operations of the CG on libpscuda kernels:
per-(l, m) 3x3 products (Sigma, C^-1, with optional beam scales) and the CG's
m-weighted inner product (polyspec/weighting.py:255), for complex128 vectors
[B, 3, nlm] on the device."""
import ctypes

import torch

from . import _lib


def _vp(t):
    return ctypes.c_void_p(t.data_ptr() if t is not None else 0)


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def real3(mat):
    """[3, 3, nlm] matrix (complex or real) as the contiguous float64 the kernels take."""
    m = mat.real if mat.is_complex() else mat
    return m.to(torch.float64).contiguous()


def matvec3(S, x, pre=None, post=None):
    """y[n, a] = post[a] * Sum_b S[a, b] * pre[b] * x[n, b]   (S float64 [3, 3, nlm])."""
    x = x.contiguous()
    y = torch.empty_like(x)
    B, nf, nlm = x.shape
    if nf != 3:
        raise ValueError("matvec3 works on [B, 3, nlm] vectors")
    _lib.call("ps_lm_matvec3", _vp(S), _vp(pre), _vp(post), _vp(x), _vp(y), B, nlm, _stream())
    return y


def dot(x, y, w):
    """Re Sum w x conj(y) over fields and lm, per batch member (w float64 [nlm])."""
    x = x.contiguous()
    y = y.contiguous()
    B, nf, nlm = x.shape
    if nf != 3:
        raise ValueError("dot works on [B, 3, nlm] vectors")
    n = ctypes.c_size_t()
    _lib.call("ps_lm_dot_workspace_bytes", B, nlm, ctypes.byref(n))
    ws = torch.empty(max(int(n.value), 8), dtype=torch.uint8, device=x.device)
    out = torch.empty(B, dtype=torch.float64, device=x.device)
    _lib.call("ps_lm_dot", _vp(x), _vp(y), _vp(w), B, nlm, _vp(out), _vp(ws), int(n.value), _stream())
    return out


def matvec3_add(S, x, y):
    """y[n, a] += Sum_b S[a, b] x[n, b] in place (S float64 [3, 3, nlm]; y contiguous, not x)."""
    x = x.contiguous()
    B, nf, nlm = x.shape
    if nf != 3 or not y.is_contiguous() or y.shape != x.shape:
        raise ValueError("matvec3_add works on contiguous [B, 3, nlm] vectors")
    _lib.call("ps_lm_matvec3_add", _vp(S), _vp(x), _vp(y), B, nlm, _stream())
    return y


def quad_dot(S, x, w):
    """Re Sum w x conj(S x) per batch member (S x is not stored)."""
    x = x.contiguous()
    B, nf, nlm = x.shape
    if nf != 3:
        raise ValueError("quad_dot works on [B, 3, nlm] vectors")
    n = ctypes.c_size_t()
    _lib.call("ps_lm_dot_workspace_bytes", B, nlm, ctypes.byref(n))
    ws = torch.empty(max(int(n.value), 8), dtype=torch.uint8, device=x.device)
    out = torch.empty(B, dtype=torch.float64, device=x.device)
    _lib.call("ps_lm_quad_dot", _vp(S), _vp(x), _vp(w), B, nlm, _vp(out), _vp(ws), int(n.value), _stream())
    return out


def xr_update(x, slot, alpha, p, r, q):
    """x[slot[n]] += alpha[n] p[n] and r[n] -= alpha[n] q[n] in place (complex128, contiguous; slot int64
    or None for the identity)."""
    B = p.shape[0]
    per = p[0].numel() if B else 0
    for t in (x, p, r, q):
        if not t.is_contiguous() or t.dtype != torch.complex128:
            raise ValueError("xr_update needs contiguous complex128 tensors")
    alpha = alpha.to(torch.float64).contiguous()
    _lib.call("ps_cg_xr_update", _vp(x), _vp(slot), _vp(alpha), _vp(p), _vp(r), _vp(q), B, per, _stream())


def direction(p, z, beta):
    """p[n] = z[n] + beta[n] p[n] in place (complex128, contiguous)."""
    B = p.shape[0]
    per = p[0].numel() if B else 0
    if not (p.is_contiguous() and z.is_contiguous()) or p.dtype != torch.complex128 or z.dtype != torch.complex128:
        raise ValueError("direction needs contiguous complex128 tensors")
    beta = beta.to(torch.float64).contiguous()
    _lib.call("ps_cg_direction", _vp(p), _vp(z), _vp(beta), B, per, _stream())
