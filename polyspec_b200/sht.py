"""Device-side HEALPix SHTs through libpscuda (torch tensors in, torch tensors out).

``SHTPlan(nside, lmax)`` wraps one ``ps_plan``.  Its transforms take and
return CUDA tensors in the ducc0 layout used by the reference
(polyspec/base.py:147-282):

* spin 0:   alm ``complex128 [B, nalm]``    <->  map ``float64 [B, npix]``
* spin s>0: alm ``complex128 [B, 2, nalm]`` <->  map ``float64 [B, 2, npix]``
  (components G, C <-> Q, U)

``adjoint`` is ducc0's ``adjoint_synthesis`` times ``scale``.

With ``autotune=True`` (default) the first call of each (direction, spin,
batch bucket) times the candidate tile shapes of the Legendre kernels and, for
``prec='mixed'``, the FP64 pipeline too (an FP64 plan is kept beside the mixed
one) and keeps the fastest (polyspec_b200.autotune; choices cached in JSON).
The tensor-core pipeline wins at large batches; for one or a few maps the FP64
CUDA-core kernels are faster (and exact to FP64).
"""
import ctypes

import torch

from . import _lib


def nalm(lmax):
    return (lmax + 1) * (lmax + 2) // 2


class SHTPlan:
    def __init__(self, nside, lmax=None, spins=(0, 1, 2, 3), prec="fp64", device=None, autotune=True):
        if not torch.cuda.is_available():
            raise RuntimeError("the CUDA backend needs a GPU (no CPU fallback)")
        self.nside = int(nside)
        self.lmax = 3 * self.nside - 1 if lmax is None else int(lmax)
        self.npix = 12 * self.nside ** 2
        self.nalm = nalm(self.lmax)
        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        self.prec = prec
        mask = 0
        for s in spins:
            mask |= 1 << int(s)
        self.spins = tuple(spins)
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _lib.call("ps_plan_create", self.nside, self.lmax, self.lmax, mask,
                      _lib.PS_PREC_FP64 if prec == "fp64" else _lib.PS_PREC_MIXED, ctypes.byref(h))
        self._h = h
        self._ws = None
        # autotuning: tile shapes of this plan and, for mixed precision, an FP64 plan
        # beside it for the small-batch path
        self._h64 = None
        self._tuner = None
        if autotune:
            from .autotune import Tuner
            handles = {"fp64" if prec == "fp64" else "mixed": h}
            if prec != "fp64":
                h64 = ctypes.c_void_p()
                with torch.cuda.device(self.device):
                    rc = _lib.lib().ps_plan_create(self.nside, self.lmax, self.lmax, mask, _lib.PS_PREC_FP64,
                                                   ctypes.byref(h64))
                # an FP64 plan may be unsupported where the mixed one is not (at Nside 2048 the
                # FP64 Bluestein work arrays exceed shared memory): tune the mixed tiles only then
                if rc == _lib.PS_OK:
                    self._h64 = h64
                    handles["fp64"] = h64
                elif rc != _lib.PS_ERR_UNSUPPORTED:
                    _lib.check("ps_plan_create", rc)
            self._tuner = Tuner(self.nside, self.lmax, handles, self.device)
        # counters of transforms issued through this plan
        self.n_synthesis = 0
        self.n_adjoint = 0

    def __del__(self):
        for name in ("_h", "_h64"):
            h = getattr(self, name, None)
            if h is not None and h.value and _lib._lib is not None:
                _lib.lib().ps_plan_destroy(h)
                setattr(self, name, None)

    # ------------------------------------------------------------ autotuning
    def _pick(self, key, run):
        """Plan handle for `key` = (direction, spin, batch); `run(handle)` issues the
        transform.  With autotuning, the first call of a key times every pipeline and
        tile shape (polyspec_b200.autotune)."""
        if self._tuner is None:
            return self._h
        direction, spin, B = key
        return self._tuner.select(0 if direction == "synthesis" else 1, spin, B, run)

    def error_flag(self, reset=True):
        """Device error flag of the plan (set by a kernel whose bounded wait expired)."""
        v = ctypes.c_int()
        _lib.call("ps_plan_error_flag", self._h, ctypes.byref(v), int(reset))
        return int(v.value)

    # ------------------------------------------------------------ workspace
    def workspace(self, batch, spin, adjoint):
        need = 0
        for h in (self._h, self._h64):
            if h is None:
                continue
            n = ctypes.c_size_t()
            _lib.call("ps_sht_workspace_bytes", h, int(batch), int(spin), int(adjoint), ctypes.byref(n))
            need = max(need, int(n.value))
        if self._ws is None or self._ws.numel() < need:
            self._ws = torch.empty(max(need, 256), dtype=torch.uint8, device=self.device)
        return self._ws, need

    @staticmethod
    def _stream():
        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def _check_alm(self, alm, spin):
        ncomp = 1 if spin == 0 else 2
        if alm.dtype != torch.complex128 or not alm.is_cuda:
            raise TypeError("alm must be a complex128 CUDA tensor")
        if alm.shape[-1] != self.nalm:
            raise ValueError("Wrong number of alm coefficients!")
        if spin > 0 and (alm.dim() < 2 or alm.shape[-2] != 2):
            raise ValueError("spin > 0 needs alm[..., 2, nalm] (G, C)")
        lead = alm.shape[:-2] if spin > 0 else alm.shape[:-1]
        B = 1
        for d in lead:
            B *= int(d)
        return lead, B, ncomp

    def synthesis(self, alm, spin=0):
        spin = int(spin)
        lead, B, ncomp = self._check_alm(alm, spin)
        alm = alm.contiguous()
        shape = tuple(lead) + ((2,) if spin > 0 else ()) + (self.npix,)
        out = torch.empty(shape, dtype=torch.float64, device=alm.device)
        if B == 0:
            return out
        ws, nbytes = self.workspace(B, spin, 0)

        def run(h):
            _lib.call("ps_synthesis", h, ctypes.c_void_p(alm.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                      B, spin, ctypes.c_void_p(ws.data_ptr()), nbytes, self._stream())
        run(self._pick(("synthesis", spin, B), run))
        self.n_synthesis += B
        return out

    def adjoint(self, map, spin=0, scale=1.0):
        spin = int(spin)
        if map.dtype != torch.float64 or not map.is_cuda:
            raise TypeError("map must be a float64 CUDA tensor")
        if map.shape[-1] != self.npix:
            raise ValueError("map has %d pixels, expected %d" % (map.shape[-1], self.npix))
        if spin > 0 and (map.dim() < 2 or map.shape[-2] != 2):
            raise ValueError("spin > 0 needs map[..., 2, npix] (Q, U)")
        lead = map.shape[:-2] if spin > 0 else map.shape[:-1]
        B = 1
        for d in lead:
            B *= int(d)
        map = map.contiguous()
        shape = tuple(lead) + ((2,) if spin > 0 else ()) + (self.nalm,)
        out = torch.empty(shape, dtype=torch.complex128, device=map.device)
        if B == 0:
            return out
        ws, nbytes = self.workspace(B, spin, 1)

        def run(h):
            _lib.call("ps_adjoint", h, ctypes.c_void_p(map.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                      B, spin, float(scale), ctypes.c_void_p(ws.data_ptr()), nbytes, self._stream())
        run(self._pick(("adjoint", spin, B), run))
        self.n_adjoint += B
        return out
