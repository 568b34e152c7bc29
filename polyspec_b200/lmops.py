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
