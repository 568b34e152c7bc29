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

Legendre tables (``tables='auto'``, mixed precision only): the first transform
of a spin builds the plan's FP32 Legendre table of that spin
(``ps_plan_build_table``) when it fits in ``table_fraction`` of the free device
memory (default 0.45, or the environment variable PS_TABLE_MEM_FRACTION); the
Legendre stages of that spin then stream the table through tensor-core GEMMs.
Where it does not fit (Nside 2048 at lmax 4096 needs 137 GB for spin 0) the
on-the-fly kernels run.  ``tables=True`` builds regardless of the budget (and
raises if the allocation fails), ``tables=False`` never builds.
"""
import ctypes
import os

import torch

from . import _lib


def nalm(lmax):
    return (lmax + 1) * (lmax + 2) // 2


class SHTPlan:
    def __init__(self, nside, lmax=None, spins=(0, 1, 2, 3), prec="fp64", device=None, autotune=True,
                 tables="auto", table_fraction=None, table_format=None):
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
        # Legendre table format of a mixed plan: 'tf32x3' (FP32 values, split by the kernels) or
        # 'bf16x3' (BF16 hi + mid + lo planes in the tensor core's operand layout, 1.5x the bytes)
        if table_format is None:
            table_format = os.environ.get("PS_TABLE_FORMAT", "tf32x3")
        if table_format not in ("tf32x3", "bf16x3"):
            raise ValueError("table_format must be 'tf32x3' or 'bf16x3'")
        self.table_format = table_format
        if prec != "fp64":
            _lib.call("ps_plan_set_table_format", h, 1 if table_format == "bf16x3" else 0)
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
        # Legendre tables: spins already tried (built or refused)
        self.tables = tables if prec != "fp64" else False
        self.table_fraction = float(table_fraction if table_fraction is not None
                                    else os.environ.get("PS_TABLE_MEM_FRACTION", 0.45))
        self._tab_tried = set()

    # ------------------------------------------------------------ Legendre tables
    def table_bytes(self, spin):
        n = ctypes.c_size_t()
        _lib.call("ps_plan_table_bytes", self._h, int(spin), ctypes.byref(n))
        return int(n.value)

    def has_table(self, spin):
        v = ctypes.c_int()
        _lib.call("ps_plan_has_table", self._h, int(spin), ctypes.byref(v))
        return bool(v.value)

    def build_table(self, spin, force=False):
        """Build the FP32 Legendre table of `spin` (mixed plans).  Without `force`, only when
        it fits in table_fraction of the free device memory; returns whether the plan has it."""
        spin = int(spin)
        if self.prec == "fp64":
            return False
        if self.has_table(spin):
            return True
        need = self.table_bytes(spin)
        with torch.cuda.device(self.device):
            free, _ = torch.cuda.mem_get_info()
            if not force and need > self.table_fraction * free:
                torch.cuda.empty_cache()
                free, _ = torch.cuda.mem_get_info()
                if need > self.table_fraction * free:
                    return False
            rc = _lib.lib().ps_plan_build_table(self._h, spin, self._stream())
            if rc == _lib.PS_ERR_NOMEM:
                torch.cuda.empty_cache()
                rc = _lib.lib().ps_plan_build_table(self._h, spin, self._stream())
            if rc == _lib.PS_ERR_NOMEM and not force:
                return False
            _lib.check("ps_plan_build_table", rc)
        return True

    def drop_tables(self):
        _lib.call("ps_plan_drop_tables", self._h)
        self._tab_tried.clear()

    def _maybe_table(self, spin):
        if self.tables is False or spin in self._tab_tried:
            return
        self._tab_tried.add(spin)
        self.build_table(spin, force=self.tables is True)

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
        table = self.prec != "fp64" and self.has_table(spin)
        return self._tuner.select(0 if direction == "synthesis" else 1, spin, B, run, table=table)

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
        self._maybe_table(spin)
        ws, nbytes = self.workspace(B, spin, 0)

        def run(h):
            _lib.call("ps_synthesis", h, ctypes.c_void_p(alm.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                      B, spin, ctypes.c_void_p(ws.data_ptr()), nbytes, self._stream())
        run(self._pick(("synthesis", spin, B), run))
        self.n_synthesis += B
        return out

    def weighted_roundtrip(self, alm, weight, lscale=None, scale=1.0, out=None):
        """Fused  out = scale * lscale * Y^H W Y (lscale * alm)  for every field of alm [B, nf, nalm]
        (nf = 1: T, spin 0; nf = 3: T spin 0 and (E, B) spin 2), weight [nf, npix] float64,
        lscale [nf, nalm] float64 or None (ps_sht_weighted_roundtrip: the maps stay in shared
        memory).  Returns None when a spin lacks its Legendre table (the caller composes
        synthesis, weight and adjoint instead)."""
        if self.prec == "fp64" or alm.dim() != 3 or alm.shape[1] not in (1, 3):
            return None
        B, nf = alm.shape[0], alm.shape[1]
        spins = [(0, 0)] if nf == 1 else [(0, 0), (2, 1)]
        for spin, _ in spins:
            self._maybe_table(spin)
            if not self.has_table(spin):
                return None
        alm = alm.contiguous()
        if out is None:
            out = torch.empty_like(alm)
        w = weight.contiguous()
        ls = lscale.contiguous() if lscale is not None else None
        for spin, c0 in spins:
            n = ctypes.c_size_t()
            _lib.call("ps_roundtrip_workspace_bytes", self._h, B, spin, ctypes.byref(n))
            if self._ws is None or self._ws.numel() < n.value:
                self._ws = torch.empty(max(n.value, 256), dtype=torch.uint8, device=self.device)
            off = c0 * self.nalm * 16
            _lib.call("ps_sht_weighted_roundtrip", self._h, ctypes.c_void_p(alm.data_ptr() + off),
                      ctypes.c_void_p(out.data_ptr() + off), nf * self.nalm, B, spin,
                      ctypes.c_void_p(w.data_ptr() + c0 * self.npix * 8),
                      ctypes.c_void_p(ls.data_ptr() + c0 * self.nalm * 8) if ls is not None else ctypes.c_void_p(0),
                      float(scale), ctypes.c_void_p(self._ws.data_ptr()), self._ws.numel(), self._stream())
        self.n_synthesis += B * len(spins)
        self.n_adjoint += B * len(spins)
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
        self._maybe_table(spin)
        ws, nbytes = self.workspace(B, spin, 1)

        def run(h):
            _lib.call("ps_adjoint", h, ctypes.c_void_p(map.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                      B, spin, float(scale), ctypes.c_void_p(ws.data_ptr()), nbytes, self._stream())
        run(self._pick(("adjoint", spin, B), run))
        self.n_adjoint += B
        return out
