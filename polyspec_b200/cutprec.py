"""Masked-band ("cut") preconditioner for the CG S^-1 filter: the exact inverse,
per order m, of the filter's operator with the masked equatorial band modelled
exactly (no counterpart in the reference, whose CG offers 'harmonic' and
'pseudo_inverse', polyspec/weighting.py:301-324).

The CG solves A x = b with A = C^-1 + B Y^H W Y B (weighting.py:297-299: Y the
synthesis, W = mask^2 N^-1 per pixel, B the beam).  The harmonic preconditioner
Sigma = (C^-1 + B^2 / N_iso)^-1 (weighting.py:76-78) treats the sky as full and
the noise as white; the masked band |b| < b_cut, fully masked rings around the
equator, is what makes CG slow: its modes couple every l of an order m.  With
Y_c the synthesis restricted to those rings and w the full-sky pixel weight that
Sigma assumes (1 / mean noise, per field),

    A  ~=  Sigma^-1 - B Y_c^H w Y_c B                                   (per m)
    M   =  Sigma + Sigma B L^H Om^1/2 K_m^-1 Om^1/2 L B Sigma,
    K_m =  I - Om^1/2 L B Sigma B L^H Om^1/2                            (Woodbury)

where L is the Legendre synthesis stage on the band's rings (the m-th Fourier
coefficient of each ring), L^H its exact adjoint, and Om = n_phi w on those rings
(Y_c^H w Y_c = L^H Om L for one m).  K_m is 3 R x 3 R (T, Q, U on R band rings)
for every m; it is built once, by applying the operator to unit vectors of the
band's phase space (all m at once: the operator is diagonal in m), and inverted
with a batched Cholesky factorisation (the band stages in FP64 for this).
Applying M costs a band-restricted Legendre synthesis and adjoint in the plan's
precision (R / (4 Nside) of a full transform's Legendre work) and one batched
matrix product per CG step.  Holes outside the band and
the quadrature error of the HEALPix grid are left to the CG.

M is symmetric positive definite whenever the model is (K_m positive definite),
so the reference's PCG update applies unchanged; orders whose K_m fails the
Cholesky factorisation fall back to Sigma.
"""
import ctypes

import numpy as np
import torch

from . import _lib, lmops


def _vp(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def ring_ranges(nside):
    """(start pixel, number of pixels) of each of the 4 nside - 1 RING-scheme rings."""
    R = 4 * nside - 1
    starts = np.zeros(R, dtype=np.int64)
    counts = np.zeros(R, dtype=np.int64)
    npix = 12 * nside * nside
    for i in range(1, R + 1):
        if i < nside:
            n, s = 4 * i, 2 * i * (i - 1)
        elif i <= 3 * nside:
            n, s = 4 * nside, 2 * nside * (nside - 1) + (i - nside) * 4 * nside
        else:
            j = 4 * nside - i
            n, s = 4 * j, npix - 2 * j * (j + 1)
        starts[i - 1], counts[i - 1] = s, n
    return starts, counts


class CutPreconditioner:
    def __init__(self, weightings, chunk=64, dtype=torch.complex64, native=None, planes=2):
        W = weightings
        base = W.base
        if not base.pol:
            raise ValueError("the cut preconditioner works on T, E, B (pol=True)")
        self.W, self.base = W, base
        dev = base.device
        nside, lmax = base.Nside, base.lmax
        # fully masked rings nearest the equator (all fields, ring and mirror)
        starts, counts = ring_ranges(nside)
        wnw = W.d_WNW
        Rh = 2 * nside
        k = 0
        for rp in range(Rh - 1, -1, -1):
            ok = True
            for r in (rp, 4 * nside - 2 - rp):
                s, n = int(starts[r]), int(counts[r])
                if float(wnw[:, s:s + n].abs().max()) != 0.0:
                    ok = False
            if not ok:
                break
            k += 1
        self.nband = k
        self.enabled = k > 0
        if not self.enabled:
            return
        P = base.plan(lmax)
        self._plan = P  # keeps the parent plans alive
        # the set-up runs the band stages in FP64 (K_m is ill-conditioned where the
        # band matters most); the per-step application in the plan's precision
        h_setup = P._h64 if P._h64 is not None else None
        self._own64 = None
        if h_setup is None and base.prec == "fp64":
            h_setup = P._h
        if h_setup is None:
            h_setup = ctypes.c_void_p()
            _lib.call("ps_plan_create", nside, lmax, lmax, 0b101, _lib.PS_PREC_FP64, ctypes.byref(h_setup))
            self._own64 = h_setup
        self._band64 = ctypes.c_void_p()
        _lib.call("ps_plan_band", h_setup, k, ctypes.byref(self._band64))
        self._band = ctypes.c_void_p()
        _lib.call("ps_plan_band", P._h, k, ctypes.byref(self._band))
        self._use = self._band64
        self.Rb = 2 * k - 1
        self.M = lmax + 1
        self.nalm = P.nalm
        band_rings = np.concatenate([np.arange(Rh - k, Rh), 4 * nside - 2 - np.arange(Rh - 2, Rh - k - 1, -1)])
        nphi = counts[band_rings].astype(np.float64)
        wbar = np.array([1.0 / np.mean(np.asarray(W.noise_cov)[f][np.asarray(W.mask)[f] > 0.99]) for f in range(3)])
        # Om^1/2 per band coordinate j = (field, ring): T rings, then Q rings, then U rings
        om = np.concatenate([nphi * wbar[0], nphi * wbar[1], nphi * wbar[2]])
        self.om_half = torch.as_tensor(np.sqrt(om), device=dev)
        self.beam = base.dev('beam_lm')           # [3, nlm]
        self.sigma_r = W.real3('Sigma')            # [3, 3, nlm] float64
        self.m0 = torch.as_tensor(base.m_arr == 0, device=dev)
        self.dtype = dtype
        self._build(chunk)
        self._use = self._band
        # one native call per application (ps_cutprec_apply: band stages on the plan's Legendre
        # tables, K_m^-1 on the tensor cores in BF16 (planes=1) or BF16 hi + lo (planes=2)) when
        # the plan is mixed with both tables; the torch composition below otherwise.  Measured at
        # Nside 1024 (6 systems to 1e-8): planes=2 takes the CG steps of the complex64 product
        # (55), planes=1 costs 15 % more (63)
        self._native = None
        self.planes = planes
        if native is not False and base.prec != "fp64" and dtype == torch.complex64:
            for spin in (0, 2):
                P._maybe_table(spin)
            h = ctypes.c_void_p()
            rc = _lib.lib().ps_cutprec_create(P._h, self._band, _vp(self.Kinv), 3 * self.Rb, int(planes),
                                              _vp(self.om_half), _vp(self.sigma_r), _vp(self.beam), _stream(),
                                              ctypes.byref(h))
            if rc == _lib.PS_OK:
                self._native = h
                self._nws = None
                torch.cuda.current_stream().synchronize()
                self.Kinv = None  # the object holds its own BF16 copy
            elif native:
                _lib.check("ps_cutprec_create", rc)

    def __del__(self):
        h = getattr(self, "_native", None)
        if h is not None and h.value and _lib._lib is not None:
            _lib.lib().ps_cutprec_destroy(h)
            self._native = None
        for name in ("_band", "_band64", "_own64"):
            h = getattr(self, name, None)
            if h is not None and h.value and _lib._lib is not None:
                _lib.lib().ps_plan_destroy(h)
                setattr(self, name, None)

    # ---------------------------------------------------------------- band Legendre stages
    def _ws(self, B, spin, adj):
        n = ctypes.c_size_t()
        _lib.call("ps_legendre_workspace_bytes", self._use, B, spin, adj, ctypes.byref(n))
        return torch.empty(max(int(n.value), 256), dtype=torch.uint8, device=self.base.device), int(n.value)

    def synth(self, alm, spin):
        """alm [B, ncomp, nalm] complex128 -> band phases [Rb, M, B, ncomp]."""
        B, nc = alm.shape[0], alm.shape[1]
        out = torch.empty((self.Rb, self.M, B, nc), dtype=torch.complex128, device=alm.device)
        ws, nb = self._ws(B, spin, 0)
        alm = alm.contiguous()  # held until the launch
        _lib.call("ps_legendre_synthesis", self._use, _vp(alm), _vp(out), B, spin, _vp(ws), nb, _stream())
        return out

    def adjoint(self, phase, spin):
        """band phases [Rb, M, B, ncomp] -> alm [B, ncomp, nalm]."""
        B, nc = phase.shape[2], phase.shape[3]
        out = torch.empty((B, nc, self.nalm), dtype=torch.complex128, device=phase.device)
        ws, nb = self._ws(B, spin, 1)
        phase = phase.contiguous()  # held until the launch
        _lib.call("ps_legendre_adjoint", self._use, _vp(phase), _vp(out), B, spin, 1.0, _vp(ws), nb, _stream())
        return out

    def _to_band(self, alm):
        """L B: alm [B, 3, nalm] -> band vector [M, 3 Rb, B] (T rings, Q rings, U rings), times Om^1/2."""
        x = alm * self.beam[None]
        p0 = self.synth(x[:, :1], 0)[..., 0]          # [Rb, M, B]
        p2 = self.synth(x[:, 1:], 2)                  # [Rb, M, B, 2]
        y = torch.cat([p0, p2[..., 0], p2[..., 1]], dim=0)  # [3 Rb, M, B]
        y = y * self.om_half[:, None, None]
        return y.permute(1, 0, 2).contiguous()

    def _from_band(self, y):
        """L^H: band vector [M, 3 Rb, B] (times Om^1/2) -> alm [B, 3, nalm] (before the beam)."""
        y = y.permute(1, 0, 2) * self.om_half[:, None, None]  # [3 Rb, M, B]
        Rb = self.Rb
        p0 = y[:Rb].unsqueeze(-1).contiguous()
        p2 = torch.stack([y[Rb:2 * Rb], y[2 * Rb:]], dim=-1).contiguous()
        a0 = self.adjoint(p0, 0)
        a2 = self.adjoint(p2, 2)
        return torch.cat([a0, a2], dim=1)  # the beam factor is applied by the caller

    def _sigma(self, alm, pre=None):
        return lmops.matvec3(self.sigma_r, alm, pre=pre)

    # ---------------------------------------------------------------- set-up
    def _build(self, chunk):
        n = 3 * self.Rb
        dev = self.base.device
        G = torch.empty((self.M, n, n), dtype=torch.complex128, device=dev)
        for j0 in range(0, n, chunk):
            nb = min(chunk, n - j0)
            e = torch.zeros((self.M, n, nb), dtype=torch.complex128, device=dev)
            idx = torch.arange(nb, device=dev)
            e[:, j0 + idx, idx] = 1.0
            col = self._to_band(self._sigma(self._from_band(e), pre=self.beam))  # [M, n, nb]
            G[:, :, j0:j0 + nb] = col
            del e, col
        # K_m = I - Herm(G_m), factorised and inverted in groups of orders (bounded memory)
        eye = torch.eye(n, dtype=torch.complex128, device=dev)
        self.Kinv = torch.empty((self.M, n, n), dtype=self.dtype, device=dev)
        self.n_bad = 0
        for m0 in range(0, self.M, 128):
            g = G[m0:m0 + 128]
            K = eye[None] - 0.5 * (g + g.conj().transpose(1, 2))
            Lc, info = torch.linalg.cholesky_ex(K)
            bad = info != 0
            self.n_bad += int(bad.sum())
            Lc[bad] = eye
            Ki = torch.cholesky_inverse(Lc)
            Ki[bad] = 0.0
            self.Kinv[m0:m0 + 128] = Ki.to(self.dtype)
            del K, Lc, Ki
        del G

    # ---------------------------------------------------------------- application
    def apply(self, r):
        """M r for r complex128 [B, 3, nlm]."""
        if self.enabled and self._native is not None:
            r = r.contiguous()
            B = r.shape[0]
            out = torch.empty_like(r)
            n = ctypes.c_size_t()
            _lib.call("ps_cutprec_workspace_bytes", self._native, B, ctypes.byref(n))
            if self._nws is None or self._nws.numel() < n.value:
                self._nws = None
                self._nws = torch.empty(int(n.value), dtype=torch.uint8, device=r.device)
            _lib.call("ps_cutprec_apply", self._native, _vp(r), _vp(out), B, _vp(self._nws), self._nws.numel(),
                      _stream())
            return out
        s = self._sigma(r)
        if not self.enabled:
            return s
        y = self._to_band(s)                                   # [M, n, B]
        w = torch.bmm(self.Kinv, y.to(self.dtype)).to(torch.complex128)
        c = self._sigma(self._from_band(w), pre=self.beam)
        c[:, :, self.m0] = c[:, :, self.m0].real.to(torch.complex128)
        return s + c
