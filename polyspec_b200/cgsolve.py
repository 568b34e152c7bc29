"""The masked CG of the optimal S^-1 filter as one native call (ps_cg_solve).

NativeCG binds a Weightings' operator arrays to a ps_cg object and solves
A x = b with A = C^-1 + B Y^H W N^-1 W Y B / A_pix and the harmonic preconditioner
Sigma: the reference's CGD with preconditioner='harmonic' (polyspec/weighting.py:
217-367) run for a batch of right-hand sides, each stopped by its own test
err = r^T Sigma r / b^T Sigma b < thresh (CGD.run, weighting.py:354-362).  The
whole loop, scalars included, runs in libpscuda; Python only passes pointers."""
import ctypes

import numpy as np
import torch

from . import _lib


def _vp(t):
    return ctypes.c_void_p(t.data_ptr() if t is not None else 0)


class NativeCG:
    def __init__(self, weightings):
        W = weightings
        base = W.base
        if not hasattr(W, 'd_WNW'):
            raise ValueError("NativeCG needs a Weightings with a noise covariance")
        self.nf = 3 if W.pol else 1
        self.plan = base.plan()
        for spin in ((0, 2) if W.pol else (0,)):
            self.plan._maybe_table(spin)
        # arrays the ps_cg object reads; kept alive here for its lifetime
        self.inv_cl = W.d_inv_Cl.real.to(torch.float64).contiguous()
        self.sigma = W.d_Sigma.real.to(torch.float64).contiguous()
        self.beam = base.dev('beam_lm').real.to(torch.float64).contiguous()
        self.weight = (W.d_WNW / W.pixel_area).to(torch.float64).expand(self.nf, -1).contiguous()
        self.nalm = int(self.plan.nalm)
        h = ctypes.c_void_p()
        _lib.call("ps_cg_create", self.plan._h, self.nf, _vp(self.inv_cl), _vp(self.sigma), _vp(self.beam),
                  _vp(self.weight), float(np.pi / (3. * base.Nside ** 2)), ctypes.byref(h))
        self._h = h
        self._ws = None

    def solve(self, b, x0=None, nstep=25, thresh=1e-4):
        """x = x0 + CG solution of A x = b for b [B, nf, nlm] complex128 on the device.  Returns
        (x, iters [B] int, err [B] float, converged: bool)."""
        b = b.to(torch.complex128).contiguous()
        B = b.shape[0]
        if b.dim() != 3 or b.shape[1] != self.nf or b.shape[2] != self.nalm:
            raise ValueError("b must be [B, %d, %d]" % (self.nf, self.nalm))
        x = torch.empty_like(b)
        if x0 is not None:
            x0 = x0.to(torch.complex128).contiguous()
            if x0.shape != b.shape:
                raise ValueError("x0 must have the shape of b")
        n = ctypes.c_size_t()
        _lib.call("ps_cg_workspace_bytes", self._h, B, ctypes.byref(n))
        if self._ws is None or self._ws.numel() < n.value:
            self._ws = torch.empty(int(n.value), dtype=torch.uint8, device=b.device)
        iters = (ctypes.c_int * B)()
        err = (ctypes.c_double * B)()
        rc = _lib.lib().ps_cg_solve(self._h, _vp(b), _vp(x0), _vp(x), B, int(nstep), float(thresh), iters, err,
                                    _vp(self._ws), self._ws.numel(),
                                    ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        if rc not in (_lib.PS_OK, _lib.PS_ERR_NOT_CONVERGED):
            _lib.check("ps_cg_solve", rc)
        return x, np.array(iters[:], dtype=np.int64), np.array(err[:]), rc == _lib.PS_OK

    def __del__(self):
        h = getattr(self, '_h', None)
        if h is not None and h.value and _lib._lib is not None:
            _lib.lib().ps_cg_destroy(h)
            self._h = None
