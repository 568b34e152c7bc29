"""Pixel-space products, radial sums and harmonic weightings on the GPU.

Mirrors the reference's Cython kernels with the same names and argument
meaning:

* ``tauNL_utils`` -- the class of polyspec/cython/tauNL_utils.pyx:21-405
  (``apply_fl_weights``, the ``multiply*`` products, ``radial_sum(_spin1)``
  and the ``gnl_*`` radial pixel sums);
* module functions ``r2c``, ``r2cstar``, ``multiplyRC(star)(_sym)``,
  ``multiplyRR(_sym)``, ``lens_phi_sum(_sym)`` and ``outer_product`` of
  polyspec/cython/ideal_fisher.pyx:18-460.

Arrays may be numpy arrays (copied to the device; results come back as numpy
arrays, as the reference returns them) or CUDA tensors (results stay CUDA
tensors).  The ``nthreads`` arguments are accepted and ignored.  Every call
runs a libpscuda kernel; there is no CPU path.
"""
import ctypes

import numpy as np
import torch

from . import _lib

_OP = {name: i for i, name in enumerate(_lib.PIX_OPS)}
_SUM = {name: i for i, name in enumerate(_lib.SUM_KINDS)}


def _dev():
    if not torch.cuda.is_available():
        raise RuntimeError("the CUDA backend needs a GPU (no CPU fallback)")
    return torch.device("cuda", torch.cuda.current_device())


def _prep(x, dtype):
    """CUDA tensor of `dtype` (contiguous) and whether the caller passed torch tensors."""
    if isinstance(x, torch.Tensor):
        return x.to(device=_dev() if not x.is_cuda else x.device, dtype=dtype).contiguous(), True
    return torch.as_tensor(np.ascontiguousarray(x), dtype=dtype, device=_dev()), False


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptrs(ts):
    arr = (ctypes.c_void_p * max(len(ts), 1))()
    for i, t in enumerate(ts):
        arr[i] = t.data_ptr()
    return arr


def _ret(t, as_torch):
    return t if as_torch else t.cpu().numpy()


def _product(op, args, kinds, out_complex, fac=0.0, npol=1, out_shape=None):
    """Run elementwise product `op` over inputs of identical shape ('r' float64, 'c' complex128)."""
    ts, flags = [], []
    for a, k in zip(args, kinds):
        t, f = _prep(a, torch.complex128 if k == "c" else torch.float64)
        ts.append(t)
        flags.append(f)
    shape = ts[0].shape
    for t in ts[1:]:
        if t.shape != shape:
            raise ValueError("all maps of a product must have the same shape")
    if out_shape is None:
        out_shape = shape
        n = ts[0].numel()
    else:
        n = int(np.prod(out_shape))
    out = torch.empty(out_shape, dtype=torch.complex128 if out_complex else torch.float64, device=ts[0].device)
    _lib.call("ps_pix_product", _OP[op], _ptrs(ts), len(ts), ctypes.c_void_p(out.data_ptr()), n, npol,
              float(fac), _stream())
    return _ret(out, all(flags))


def _radial_sum(kind, r_weights, tau, maps, kinds):
    ts, flags = [], []
    for a, k in zip(maps, kinds):
        t, f = _prep(a, torch.complex128 if k == "c" else torch.float64)
        ts.append(t)
        flags.append(f)
    nr, npix = ts[0].shape
    for t in ts[1:]:
        if tuple(t.shape) != (nr, npix):
            raise ValueError("all maps of a radial sum must have shape [nr, npix]")
    w, _ = _prep(r_weights, torch.float64)
    if w.numel() < nr:
        raise ValueError("r_weights shorter than the number of radial samples")
    tt = None
    if tau is not None:
        tt, _ = _prep(tau, torch.float64)
    nb = ctypes.c_size_t()
    _lib.call("ps_pix_radial_sum_workspace_bytes", nr, npix, ctypes.byref(nb))
    ws = torch.empty(max(int(nb.value), 8), dtype=torch.uint8, device=ts[0].device)
    out = torch.empty(1, dtype=torch.float64, device=ts[0].device)
    _lib.call("ps_pix_radial_sum", _SUM[kind], ctypes.c_void_p(w.data_ptr()),
              ctypes.c_void_p(tt.data_ptr() if tt is not None else 0), _ptrs(ts), len(ts), nr, npix,
              ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(ws.data_ptr()), int(nb.value), _stream())
    return float(out.item())


class tauNL_utils:
    """GPU mirror of polyspec/cython/tauNL_utils.pyx:21-78 (constructor) and its kernels.

    Only ``ls`` (the l of every lm of the harmonic arrays) enters the kernels
    built here; the other constructor arguments are kept for the interface.
    """

    def __init__(self, nthreads, nr, l_arr, m_arr, Lmin, Lmax, ls, ms, Ls, Ms, nmax_F):
        self.nthreads = nthreads
        self.nr = int(nr)
        self.l_arr = np.asarray(l_arr, dtype=np.int32)
        self.m_arr = np.asarray(m_arr, dtype=np.int32)
        self.Lmin, self.Lmax = int(Lmin), int(Lmax)
        self.ls = np.asarray(ls, dtype=np.int32)
        self.ms = np.asarray(ms, dtype=np.int32)
        self.Ls = np.asarray(Ls, dtype=np.int32)
        self.Ms = np.asarray(Ms, dtype=np.int32)
        self.nmax_F = nmax_F
        self.lmin, self.lmax = int(self.ls.min()), int(self.ls.max())
        self._d_ls = torch.as_tensor(self.ls, device=_dev())

    # ---------------------------------------------------------------- harmonic weightings
    def apply_fl_weights(self, flX, h_lm, weight):
        """out[r, lm] = weight Sum_X flX[l, X, r] h_lm[X, lm]   (tauNL_utils.pyx:80-98)."""
        f, as_torch = _prep(flX, torch.float64)
        h, _ = _prep(h_lm, torch.complex128)
        lsize, npol, nr = f.shape
        nlm = h.shape[1]
        if nlm > len(self.ls) or h.shape[0] < npol:
            raise ValueError("h_lm does not match flX / ls")
        out = torch.empty((nr, nlm), dtype=torch.complex128, device=h.device)
        _lib.call("ps_apply_fl_weights", ctypes.c_void_p(f.data_ptr()), lsize, npol, nr,
                  ctypes.c_void_p(h.data_ptr()), ctypes.c_void_p(self._d_ls.data_ptr()), nlm, float(weight),
                  ctypes.c_void_p(out.data_ptr()), _stream())
        return _ret(out, as_torch)

    def _radial(self, lm_map, r_weights, flXs, spin1):
        m, as_torch = _prep(lm_map, torch.complex128)
        w, _ = _prep(r_weights, torch.float64)
        f, _ = _prep(flXs, torch.float64)
        lsize, npol, nrf = f.shape
        nr, nlm = (m.shape[1], m.shape[2]) if spin1 else (m.shape[0], m.shape[1])
        if nr > nrf or w.numel() < nr or nlm > len(self.ls):
            raise ValueError("lm_map does not match r_weights / flXs / ls")
        if nrf != nr:  # the kernel indexes flXs[l][X][r] with the map's radial count
            f = f[:, :, :nr].contiguous()
        out = torch.empty((npol, nlm), dtype=torch.complex128, device=m.device)
        _lib.call("ps_radial_sum_lm", ctypes.c_void_p(m.data_ptr()), int(spin1), ctypes.c_void_p(w.data_ptr()),
                  ctypes.c_void_p(f.data_ptr()), lsize, npol, nr, ctypes.c_void_p(self._d_ls.data_ptr()), nlm,
                  ctypes.c_void_p(out.data_ptr()), _stream())
        return _ret(out, as_torch)

    def radial_sum(self, lm_map, r_weights, flXs):
        """out[X, lm] = Sum_r lm_map[r, lm] flXs[l, X, r] w_r   (tauNL_utils.pyx:220-237)."""
        return self._radial(lm_map, r_weights, flXs, False)

    def radial_sum_spin1(self, lm_map, r_weights, flXs):
        """out[X, lm] = 1/2 Sum_r (lm_map[0, r, lm] - lm_map[1, r, lm]) flXs[l, X, r] w_r  (:240-255)."""
        return self._radial(lm_map, r_weights, flXs, True)

    # ---------------------------------------------------------------- local tauNL contractions
    def _tau_tables(self):
        if not hasattr(self, '_d_tau_L'):
            L = self.Ls.astype(np.int64)
            lm_L = np.where((L >= self.Lmin) & (L <= self.Lmax), L, -1).astype(np.int32)
            self._d_tau_L = torch.as_tensor(lm_L, device=_dev())
            self._d_tau_w = torch.as_tensor(np.where(self.Ms == 0, 1., 2.), device=_dev())
            # position of each Ls entry in the l <= max(Ls) list (L_indices of tauNL_utils.pyx:50-62)
            nLmax, nLmin = int(self.Ls.max()), int(self.Ls.min())
            full = self.l_arr[self.l_arr <= nLmax]
            self._tau_pos = np.where(lm_L >= 0, np.nonzero(full >= nLmin)[0], -1)
        return self._d_tau_L, self._d_tau_w, self._tau_pos

    def tau_sum_n0(self, _arr1, _arr2, _FLLs, _r_weights, n1):
        """Sum over mu, (L, M) with Lmin <= L <= Lmax and (r, r') of m_w F_L(r, r') w_r w_r' Re(arr1 conj(arr2))
        / sqrt(4 pi) / sqrt(2 n1 + 1), arrays [n_mu, len(Ls), N_r] (tauNL_utils.pyx:604-647)."""
        lm_L, lm_w, _ = self._tau_tables()
        a1, _ = _prep(_arr1, torch.complex128)
        a2, _ = _prep(_arr2, torch.complex128)
        F, _ = _prep(_FLLs, torch.float64)
        out = 0.
        for mu in range(a1.shape[0]):
            out += tau_convolve_F(a2[mu].T.contiguous(), lm_L, F, _r_weights, A=a1[mu].T.contiguous(), lm_w=lm_w)
        return out / np.sqrt(2. * n1 + 1.)

    def _row_tables(self):
        if not hasattr(self, '_d_rows'):
            d = _dev()
            nLmax, nLmin = int(self.Ls.max()), int(self.Ls.min())
            full_l = self.l_arr[self.l_arr <= nLmax]
            row_of_full = -np.ones(len(full_l), dtype=np.int32)
            row_of_full[np.nonzero(full_l >= nLmin)[0]] = np.arange(len(self.Ls), dtype=np.int32)
            self._d_rows = (nLmax, torch.as_tensor(row_of_full, device=d),
                            torch.as_tensor(self.Ls.astype(np.int32), device=d),
                            torch.as_tensor(self.Ms.astype(np.int32), device=d),
                            torch.as_tensor(self._tau_tables()[2].astype(np.int32), device=d))
        return self._d_rows

    def _gaunt_rows(self, n):
        """Device table of the rows' Gaunt coefficients for momentum n (ps_gaunt_row_table), kept per n."""
        if not hasattr(self, '_d_gtab'):
            self._d_gtab = {}
        if n not in self._d_gtab:
            _, _, rowL, rowM, _ = self._row_tables()
            t = torch.empty(len(self.Ls) * (n + 1) * (2 * n + 1) * 2, dtype=torch.float64, device=rowL.device)
            _lib.call("ps_gaunt_row_table", ctypes.c_void_p(rowL.data_ptr()), ctypes.c_void_p(rowM.data_ptr()),
                      len(self.Ls), self.Lmin, self.Lmax, int(n), ctypes.c_void_p(t.data_ptr()), _stream())
            self._d_gtab[n] = t
        return self._d_gtab[n]

    def _F_rprime_major(self, src, F):
        """F_{L,L+Delta}(r, r') as the general contractions read it, [r'][r] innermost.  The
        estimator passes the same device FLLs for every mu1 and (n1, n3, n), so the transposed
        copy of a CUDA tensor is kept and reused while that tensor is unchanged (same storage,
        shape and version counter); numpy inputs are transposed per call."""
        if not isinstance(src, torch.Tensor) or not src.is_cuda:
            return F.transpose(2, 3).contiguous()
        key = (src.data_ptr(), tuple(src.shape), tuple(src.stride()), src._version, src.dtype)
        cache = self.__dict__.setdefault('_F_T_cache', {})
        if cache.get('src') is not src or cache.get('key') != key:
            cache['src'], cache['key'] = src, key
            cache['F'] = F.transpose(2, 3).contiguous()
        return cache['F']

    def tau_sum_general(self, _arr1, _arr2, _FLLs, _r_weights, n1, n3, n):
        """tauNL_utils.pyx:650-715: the (Delta, mu), (L, M), mu1, (r, r') sum of the direction-dependent tauNL
        estimator for arrays [2n+1, len(Ls), N_r] (ps_tau_sum_general)."""
        nLmax, row_of_full, rowL, rowM, _ = self._row_tables()
        a1, _ = _prep(_arr1, torch.complex128)
        a2, _ = _prep(_arr2, torch.complex128)
        F, _ = _prep(_FLLs, torch.float64)
        w = torch.as_tensor(np.asarray(_r_weights, dtype=np.float64), device=a1.device)
        nrow, nr = len(self.Ls), a1.shape[-1]
        if (tuple(a1.shape) != (2 * n1 + 1, nrow, nr) or tuple(a2.shape) != (2 * n3 + 1, nrow, nr)
                or F.dim() != 4 or F.shape[0] % 2 != 1 or tuple(F.shape[2:]) != (nr, nr) or w.numel() != nr
                or not 0 <= self.Lmin <= self.Lmax < F.shape[1]):
            raise ValueError("tau_sum_general: arrays must be [2n1+1 / 2n3+1, len(Ls), N_r], FLLs "
                             "[2 nmax_F + 1, > Lmax, N_r, N_r], r_weights [N_r]")
        nb = ctypes.c_size_t()
        _lib.call("ps_tau_general_workspace_bytes", nrow, nr, ctypes.byref(nb))
        ws = torch.empty(max(int(nb.value), 8), dtype=torch.uint8, device=a1.device)
        out = torch.zeros(1, dtype=torch.float64, device=a1.device)
        F = self._F_rprime_major(_FLLs, F)
        _lib.call("ps_tau_sum_general", ctypes.c_void_p(a1.data_ptr()), ctypes.c_void_p(a2.data_ptr()),
                  ctypes.c_void_p(row_of_full.data_ptr()), ctypes.c_void_p(rowL.data_ptr()),
                  ctypes.c_void_p(rowM.data_ptr()), nrow, nLmax, self.Lmin, self.Lmax, ctypes.c_void_p(F.data_ptr()),
                  F.shape[1], (F.shape[0] - 1) // 2, ctypes.c_void_p(w.data_ptr()), nr, int(n1), int(n3), int(n),
                  ctypes.c_void_p(self._gaunt_rows(int(n)).data_ptr()), ctypes.c_void_p(out.data_ptr()),
                  ctypes.c_void_p(ws.data_ptr()), int(nb.value), _stream())
        return float(out.item())

    def _collider_ws(self, nrow, device):
        nb = ctypes.c_size_t()
        _lib.call("ps_tau_collider_workspace_bytes", int(nrow), ctypes.byref(nb))
        return torch.empty(max(int(nb.value), 8), dtype=torch.uint8, device=device), int(nb.value)

    def _collider_diag(self, _arr1, _arr2, _FLLs, _r_weights, pref):
        nLmax, row_of_full, rowL, rowM, _ = self._row_tables()
        a1, _ = _prep(_arr1, torch.complex128)
        a2, _ = _prep(_arr2, torch.complex128)
        F, _ = _prep(_FLLs, torch.complex128)
        w = torch.as_tensor(np.asarray(_r_weights, dtype=np.float64), device=a1.device)
        nrow, nr = len(self.Ls), a1.shape[-1]
        if (a1.dim() != 3 or a1.shape != a2.shape or tuple(a1.shape[1:]) != (nrow, nr) or F.dim() != 3
                or tuple(F.shape[1:]) != (nr, nr) or F.shape[0] <= self.Lmax or w.numel() != nr):
            raise ValueError("collider tau sum: arrays must be [nlam, len(Ls), N_r], FLLs [> Lmax, N_r, N_r]")
        ws, nb = self._collider_ws(nrow, a1.device)
        out = torch.zeros(1, dtype=torch.float64, device=a1.device)
        pref = complex(pref)
        _lib.call("ps_tau_sum_collider_diag", ctypes.c_void_p(a1.data_ptr()), ctypes.c_void_p(a2.data_ptr()),
                  a1.shape[0], ctypes.c_void_p(rowL.data_ptr()), ctypes.c_void_p(rowM.data_ptr()), nrow, self.Lmin,
                  self.Lmax, ctypes.c_void_p(F.data_ptr()), F.shape[0], ctypes.c_void_p(w.data_ptr()), nr,
                  pref.real, pref.imag, ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(ws.data_ptr()), nb,
                  _stream())
        return float(out.item())

    def tau_sum_n0_collider(self, _arr1, _arr2, _FLLs, _r_weights, pref):
        """tauNL_utils.pyx:923-964: Sum over (L, M) of w_M Sum_{r, r'} Re(pref F_L(r, r') w w' A(r) conj(B(r')))
        for the s = 0 collider arrays [1, len(Ls), N_r] and the complex F_L [nL, N_r, N_r]
        (ps_tau_sum_collider_diag)."""
        return self._collider_diag(_arr1, _arr2, _FLLs, _r_weights, pref)

    def tau_sum_nu0_collider(self, _arr1, _arr2, _FLLs, _r_weights, pref):
        """tauNL_utils.pyx:877-921: the nu_s = 0 form, the same sum over every lambda of [2s+1, len(Ls), N_r]
        (ps_tau_sum_collider_diag)."""
        return self._collider_diag(_arr1, _arr2, _FLLs, _r_weights, pref)

    def tau_sum_general_collider(self, _arr1, _arr1c, _arr2, _arr2c, _FLLs, _r_weights, nmax_F, s, beta, _coeffs):
        """tauNL_utils.pyx:723-875: the S, Delta, Lam, lam1, (L, M), (r, r') sum of the collider estimator for
        arrays [2s+1, len(Ls), N_r] (beta and its conjugate), complex F [2 nmax_F + 1, > Lmax, N_r, N_r] and the
        coupling coefficients C_S, S = 0, 2, .., 2s (ps_tau_sum_collider_general)."""
        nLmax, row_of_full, rowL, rowM, _ = self._row_tables()
        arrs = [_prep(x, torch.complex128)[0] for x in (_arr1, _arr1c, _arr2, _arr2c)]
        F, _ = _prep(_FLLs, torch.complex128)
        dev = arrs[0].device
        w = torch.as_tensor(np.asarray(_r_weights, dtype=np.float64), device=dev)
        c = torch.as_tensor(np.asarray(_coeffs, dtype=np.complex128).reshape(-1), device=dev)
        nrow, nr = len(self.Ls), arrs[0].shape[-1]
        s = int(s)
        if (any(tuple(x.shape) != (2 * s + 1, nrow, nr) for x in arrs) or F.dim() != 4
                or F.shape[0] != 2 * int(nmax_F) + 1 or tuple(F.shape[2:]) != (nr, nr) or F.shape[1] <= self.Lmax
                or w.numel() != nr or c.numel() != s + 1):
            raise ValueError("tau_sum_general_collider: arrays must be [2s+1, len(Ls), N_r], FLLs "
                             "[2 nmax_F + 1, > Lmax, N_r, N_r], coeffs [s + 1]")
        ws, nb = self._collider_ws(nrow, dev)
        out = torch.zeros(1, dtype=torch.float64, device=dev)
        real_beta = int(complex(beta).imag == 0)
        _lib.call("ps_tau_sum_collider_general", *[ctypes.c_void_p(x.data_ptr()) for x in arrs],
                  ctypes.c_void_p(rowL.data_ptr()), ctypes.c_void_p(rowM.data_ptr()), nrow, int(self.Ls.min()),
                  nLmax, self.Lmin, self.Lmax, ctypes.c_void_p(F.data_ptr()), F.shape[1], int(nmax_F),
                  ctypes.c_void_p(w.data_ptr()), nr, s, real_beta, ctypes.c_void_p(c.data_ptr()),
                  ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(ws.data_ptr()), nb, _stream())
        return float(out.item())

    def convolve_F_general(self, _PQ, _FLLs, _r_weights, out_real, out_imag, n1, n3, n, mu1, inds):
        """tauNL_utils.pyx:1069-1180: the Gaunt-weighted F convolutions for one mu1, accumulated in place into
        out_real / out_imag [len(l <= nLmax), len(inds)] (ps_convolve_F_general)."""
        nLmax, row_of_full, rowL, rowM, full_of_row = self._row_tables()
        PQ, _ = _prep(_PQ, torch.complex128)
        F, _ = _prep(_FLLs, torch.float64)
        w = torch.as_tensor(np.asarray(_r_weights, dtype=np.float64), device=PQ.device)
        ind = _i32(inds)
        o_re, _ = _prep(out_real, torch.complex128)
        o_im, _ = _prep(out_imag, torch.complex128)
        nr, nfull = len(inds), int(np.sum(self.l_arr <= nLmax))
        ia = np.asarray(inds)
        if (tuple(PQ.shape) != (2 * n3 + 1, len(self.Ls), nr) or F.dim() != 4 or F.shape[0] % 2 != 1
                or F.shape[2] != F.shape[3] or (nr and (ia.min() < 0 or ia.max() >= F.shape[2]))
                or w.numel() < nr or tuple(o_re.shape) != (nfull, nr) or tuple(o_im.shape) != (nfull, nr)
                or not 0 <= self.Lmin <= self.Lmax < F.shape[1] or abs(mu1) > n1):
            raise ValueError("convolve_F_general: PQ [2n3+1, len(Ls), len(inds)], FLLs [2 nmax_F + 1, > Lmax, "
                             "N_r, N_r] with inds < N_r, outputs [len(l <= max(Ls)), len(inds)], |mu1| <= n1")
        if nr == 0:
            return
        F = self._F_rprime_major(_FLLs, F)
        _lib.call("ps_convolve_F_general", ctypes.c_void_p(PQ.data_ptr()), ctypes.c_void_p(row_of_full.data_ptr()),
                  ctypes.c_void_p(rowL.data_ptr()), ctypes.c_void_p(rowM.data_ptr()),
                  ctypes.c_void_p(full_of_row.data_ptr()), PQ.shape[1], nLmax, self.Lmin, self.Lmax,
                  ctypes.c_void_p(F.data_ptr()), F.shape[1], F.shape[2], (F.shape[0] - 1) // 2,
                  ctypes.c_void_p(w.data_ptr()), ctypes.c_void_p(ind.data_ptr()), len(inds), int(n1), int(n3), int(n),
                  int(mu1), ctypes.c_void_p(self._gaunt_rows(int(n)).data_ptr()), ctypes.c_void_p(o_re.data_ptr()),
                  ctypes.c_void_p(o_im.data_ptr()), _stream())
        for dst, src in ((out_real, o_re), (out_imag, o_im)):
            if isinstance(dst, torch.Tensor):
                if dst.data_ptr() != src.data_ptr():
                    dst.copy_(src)
            else:
                dst[...] = src.cpu().numpy()

    def convolve_F_n0(self, PQ, cPQ, FLLs, r_weights, out_real, out_imag, n1, mu1, nmax_F, inds):
        """tauNL_utils.pyx:1026-1067 (n = 0, n1 > 0): with conv = the F_L convolution of convolve_F_n000,
        out_real = p conv(PQ) + q conv(cPQ), out_imag = p conv(PQ) - q conv(cPQ), p = (-1)^(n1-mu1) / 2 / sqrt(2n1+1),
        q = 1 / 2 / sqrt(2n1+1), written in place at the rows of the L range."""
        def conv(X):
            o = torch.zeros(tuple(out_real.shape), dtype=torch.complex128, device=_dev())
            self.convolve_F_n000(X, FLLs, r_weights, o, nmax_F, inds)
            return o
        a, b = conv(PQ), conv(cPQ)
        pp = (-1.) ** (n1 - mu1) / np.sqrt(2. * n1 + 1.) / 2.
        pm = 1. / np.sqrt(2. * n1 + 1.) / 2.
        rows = np.nonzero(self._tau_tables()[2] >= 0)[0]
        pos = torch.as_tensor(self._tau_tables()[2][rows], device=_dev())
        vr, vi = (pp * a + pm * b)[pos], (pp * a - pm * b)[pos]
        for dst, v in ((out_real, vr), (out_imag, vi)):
            if isinstance(dst, torch.Tensor):
                dst[pos.to(dst.device)] = v.to(dst.device)
            else:
                dst[self._tau_tables()[2][rows]] = v.cpu().numpy()

    def compute_pF_map_real(self, _input_plus, _input_minus, _plLXs, _r_weights, n1, mu1, nmax, lmax, _output, inds):
        """tauNL_utils.pyx:1531-1620: _output [npol, len(ls)] += the Gaunt-weighted gather of the shifted inputs
        ([nlm(lmax), len(inds)] complex) times p_{l,l+Delta}^X(r) w_r, in place (ps_pF_map_real)."""
        plus, _ = _prep(_input_plus, torch.complex128)
        minus, _ = _prep(_input_minus, torch.complex128)
        pl, _ = _prep(_plLXs, torch.float64)
        w = torch.as_tensor(np.asarray(_r_weights, dtype=np.float64), device=plus.device)
        ind = _i32(inds)
        if not hasattr(self, '_d_ms'):
            self._d_ms = torch.as_tensor(self.ms, device=_dev())
            self._d_ls32 = torch.as_tensor(self.ls, device=_dev())
        nshift, lsize, npol, nrp = pl.shape
        out, _ = _prep(_output, torch.complex128)
        _lib.call("ps_pF_map_real", ctypes.c_void_p(plus.data_ptr()), ctypes.c_void_p(minus.data_ptr()), int(lmax),
                  plus.shape[1], ctypes.c_void_p(pl.data_ptr()), nshift, lsize, npol, nrp,
                  ctypes.c_void_p(w.data_ptr()), ctypes.c_void_p(ind.data_ptr()),
                  ctypes.c_void_p(self._d_ls32.data_ptr()), ctypes.c_void_p(self._d_ms.data_ptr()), len(self.ls),
                  int(n1), int(mu1), int(nmax), ctypes.c_void_p(out.data_ptr()), _stream())
        if isinstance(_output, torch.Tensor):
            if _output.data_ptr() != out.data_ptr():
                _output.copy_(out)
        else:
            _output[...] = out.cpu().numpy()

    def compute_pF_map_complex(self, _input_plus, _input_minus, _plLXs, _r_weights, n1, mu1, nmax, lmax, _output,
                               inds):
        """tauNL_utils.pyx:1357-1446: _output [npol, len(ls)] += the Gaunt-weighted shifts of the inputs
        ([nlm(lmax), len(inds)] complex) times the complex collider p^beta_{l,l+Delta}^X(r) w_r, in place
        (ps_pF_map_complex); -n1 <= mu1 <= n1."""
        plus, _ = _prep(_input_plus, torch.complex128)
        minus, _ = _prep(_input_minus, torch.complex128)
        pl, _ = _prep(_plLXs, torch.complex128)
        w = torch.as_tensor(np.asarray(_r_weights, dtype=np.float64), device=plus.device)
        ind = _i32(inds)
        if not hasattr(self, '_d_ms'):
            self._d_ms = torch.as_tensor(self.ms, device=_dev())
            self._d_ls32 = torch.as_tensor(self.ls, device=_dev())
        nshift, lsize, npol, nrp = pl.shape
        out, _ = _prep(_output, torch.complex128)
        _lib.call("ps_pF_map_complex", ctypes.c_void_p(plus.data_ptr()), ctypes.c_void_p(minus.data_ptr()),
                  int(lmax), plus.shape[1], ctypes.c_void_p(pl.data_ptr()), nshift, lsize, npol, nrp,
                  ctypes.c_void_p(w.data_ptr()), ctypes.c_void_p(ind.data_ptr()),
                  ctypes.c_void_p(self._d_ls32.data_ptr()), ctypes.c_void_p(self._d_ms.data_ptr()), len(self.ls),
                  int(n1), int(mu1), int(nmax), ctypes.c_void_p(out.data_ptr()), _stream())
        if isinstance(_output, torch.Tensor):
            if _output.data_ptr() != out.data_ptr():
                _output.copy_(out)
        else:
            _output[...] = out.cpu().numpy()

    def convolve_F_general_collider(self, PQ, cPQ, FLLs, r_weights, out_real, out_imag, s, lam1, nmax_F, S_weights,
                                    inds):
        """tauNL_utils.pyx:1197-1355: the collider F convolution for one lam1, accumulated in place into
        out_real / out_imag [len(l <= nLmax), len(inds)] (ps_convolve_F_collider)."""
        nLmax, row_of_full, rowL, rowM, full_of_row = self._row_tables()
        a, _ = _prep(PQ, torch.complex128)
        c, _ = _prep(cPQ, torch.complex128)
        F, _ = _prep(FLLs, torch.complex128)
        dev = a.device
        w = torch.as_tensor(np.asarray(r_weights, dtype=np.float64), device=dev)
        sw = torch.as_tensor(np.asarray(S_weights, dtype=np.complex128).reshape(-1), device=dev)
        ind = _i32(inds)
        nrow, nr = len(self.Ls), a.shape[-1]
        if (a.shape != c.shape or a.dim() != 3 or tuple(a.shape[1:]) != (nrow, nr) or F.dim() != 4
                or F.shape[0] != 2 * int(nmax_F) + 1 or F.shape[2] != F.shape[3] or F.shape[1] <= self.Lmax
                or ind.numel() != nr or sw.numel() != int(s) + 1):
            raise ValueError("convolve_F_general_collider: PQ, cPQ [2s+1, len(Ls), len(inds)], FLLs "
                             "[2 nmax_F + 1, > Lmax, N_r, N_r], S_weights [s + 1]")
        ore, _ = _prep(out_real, torch.complex128)
        oim, _ = _prep(out_imag, torch.complex128)
        _lib.call("ps_convolve_F_collider", ctypes.c_void_p(a.data_ptr()), ctypes.c_void_p(c.data_ptr()),
                  ctypes.c_void_p(rowL.data_ptr()), ctypes.c_void_p(rowM.data_ptr()),
                  ctypes.c_void_p(full_of_row.data_ptr()), nrow, int(self.Ls.min()), nLmax, self.Lmin, self.Lmax,
                  ctypes.c_void_p(F.data_ptr()), F.shape[1], F.shape[2], int(nmax_F), ctypes.c_void_p(w.data_ptr()),
                  ctypes.c_void_p(ind.data_ptr()), nr, int(s), int(lam1), ctypes.c_void_p(sw.data_ptr()),
                  ctypes.c_void_p(ore.data_ptr()), ctypes.c_void_p(oim.data_ptr()), _stream())
        for dst, src in ((out_real, ore), (out_imag, oim)):
            if isinstance(dst, torch.Tensor):
                if dst.data_ptr() != src.data_ptr():
                    dst.copy_(src)
            else:
                dst[...] = src.cpu().numpy()

    def convolve_F_n000_real(self, PQ, FLLs, r_weights, out, nmax_F, inds):
        """tauNL_utils.pyx:997-1023: convolve_F_n000 with the real part of a complex (collider) F."""
        F = FLLs.real.contiguous() if isinstance(FLLs, torch.Tensor) else np.ascontiguousarray(np.real(FLLs))
        self.convolve_F_n000(PQ, F, r_weights, out, nmax_F, inds)

    def shift_and_weight_map_all(self, flX, h_lm, n, mu, weight, Larr_real, Larr_imag, nmax):
        """Gaunt-weighted l-shifts of the transfer-weighted harmonics (tauNL_utils.pyx:407-512):
        Larr_real/imag [N_r, nlm(lmax + n)] += Sum over shifts Delta of the (L = l + Delta, |mu -+ m|)
        contributions, in place; two kernels (a coefficient table per (Delta, target), then a gather
        per (target, radial sample)) in ps_shift_weight_map_all."""
        f, _ = _prep(flX, torch.float64)
        h, _ = _prep(h_lm, torch.complex128)
        nshift, lsize, npol, nr = f.shape
        nsrc = h.shape[1]
        lmax_src = int(self.ls.max())
        lmax_t = lmax_src + int(n)
        if not hasattr(self, '_sw_tables') or self._sw_tables[0] != lmax_t:
            full_l = np.concatenate([np.arange(m, lmax_src + 1) for m in range(lmax_src + 1)])
            full_m = np.concatenate([np.full(lmax_src + 1 - m, m) for m in range(lmax_src + 1)])
            src_of = -np.ones(len(full_l), dtype=np.int32)
            pos = {(int(l), int(m)): i for i, (l, m) in enumerate(zip(full_l, full_m))}
            for i, (l, m) in enumerate(zip(self.ls, self.ms)):
                src_of[pos[(int(l), int(m))]] = i
            tK = np.concatenate([np.full(lmax_t + 1 - m, m) for m in range(lmax_t + 1)]).astype(np.int32)
            tL = np.concatenate([np.arange(m, lmax_t + 1) for m in range(lmax_t + 1)]).astype(np.int32)
            d = _dev()
            self._sw_tables = (lmax_t, torch.as_tensor(src_of, device=d), torch.as_tensor(tL, device=d),
                               torch.as_tensor(tK, device=d), torch.as_tensor(self.ls.astype(np.int32), device=d))
        _, d_src_of, d_tL, d_tK, d_src_l = self._sw_tables
        ntarget = d_tL.numel()
        Lre, re_torch = _prep(Larr_real, torch.complex128)
        Lim, _ = _prep(Larr_imag, torch.complex128)
        if Lre.shape != (nr, ntarget) or Lim.shape != (nr, ntarget):
            raise ValueError("Larr arrays must be [N_r, nlm(lmax + n)]")
        nb = ctypes.c_size_t()
        _lib.call("ps_shift_weight_workspace_bytes", ntarget, int(n), ctypes.byref(nb))
        ws = torch.empty(max(int(nb.value), 8), dtype=torch.uint8, device=Lre.device)
        w = complex(weight)
        _lib.call("ps_shift_weight_map_all", ctypes.c_void_p(f.data_ptr()), nshift, lsize, npol, nr,
                  ctypes.c_void_p(h.data_ptr()), nsrc, ctypes.c_void_p(d_src_l.data_ptr()),
                  ctypes.c_void_p(d_src_of.data_ptr()), lmax_src, ctypes.c_void_p(d_tL.data_ptr()),
                  ctypes.c_void_p(d_tK.data_ptr()), ntarget, int(n), int(mu), w.real, w.imag, int(nmax),
                  ctypes.c_void_p(Lre.data_ptr()), ctypes.c_void_p(Lim.data_ptr()), ctypes.c_void_p(ws.data_ptr()),
                  int(nb.value), _stream())
        for dst, src in ((Larr_real, Lre), (Larr_imag, Lim)):
            if isinstance(dst, torch.Tensor):
                if dst.data_ptr() != src.data_ptr():
                    dst.copy_(src)
            else:
                dst[...] = src.cpu().numpy()

    def convolve_F_n000(self, PQ, FLLs, r_weights, out, nmax_F, inds):
        """out[i, j] = Sum_k F_L(r_inds[j], r_inds[k]) w_k PQ[ip, k] / sqrt(4 pi) for the Ls entry ip at row i of
        the l <= nLmax list, Lmin <= L <= Lmax (tauNL_utils.pyx:966-995); out is written in place."""
        lm_L, _, pos = self._tau_tables()
        inds = np.asarray(inds, dtype=np.int64)
        F = FLLs[nmax_F] if isinstance(FLLs, torch.Tensor) else np.asarray(FLLs)[nmax_F]
        F = F[:, inds][:, :, inds]
        d_F, _ = _prep(F, torch.float64)
        X, _ = _prep(PQ.T if isinstance(PQ, torch.Tensor) else np.asarray(PQ).T, torch.complex128)
        conv = tau_convolve_F(X, lm_L, d_F, np.asarray(r_weights, dtype=np.float64)[:len(inds)])
        rows = np.nonzero(pos >= 0)[0]
        vals = conv.T[torch.as_tensor(rows, device=conv.device)]
        if isinstance(out, torch.Tensor):
            out[torch.as_tensor(pos[rows], device=out.device)] = vals.to(out.device)
        else:
            out[pos[rows]] = vals.cpu().numpy()

    # ---------------------------------------------------------------- map products
    def multiply(self, map1, map2, map3):
        return _product("multiply", (map1, map2, map3), "rrr", False)

    def multiply_asym(self, map1A, map1B, map3A, map3B):
        return _product("multiply_asym", (map1A, map1B, map3A, map3B), "rrrr", False)

    def multiplyC(self, map1, map2, map3c):
        return _product("multiplyC", (map1, map2, map3c), "rrc", True)

    def multiplyC_asym(self, map1A, map1B, map3cA, map3cB):
        return _product("multiplyC_asym", (map1A, map1B, map3cA, map3cB), "rrcc", True)

    def multiplyCC(self, map1, map2, map3c):
        return _product("multiplyCC", (map1, map2, map3c), "rrc", False)

    def multiplyCC_asym(self, map1A, map1B, map2A, map2B, map3cA, map3cB):
        return _product("multiplyCC_asym", (map1A, map1B, map2A, map2B, map3cA, map3cB), "rrrrcc", False)

    def multiply2(self, B1, B2, C1, C2):
        return _product("multiply2", (B1, B2, C1, C2), "rrcc", False)

    def multiply2R(self, A, B):
        return _product("multiply2R", (A, B), "rr", False)

    def multiply2C(self, Ac, B):
        return _product("multiply2C", (Ac, B), "cr", True)

    # ---------------------------------------------------------------- radial pixel sums
    def gnl_loc_sum(self, r_weights, P_maps, Q_maps):
        return _radial_sum("gnl_loc_sum", r_weights, None, (P_maps, Q_maps), "rr")

    def gnl_loc_disc_sum(self, r_weights, P_maps1, P_maps2, Q_maps1, Q_maps2):
        return _radial_sum("gnl_loc_disc_sum", r_weights, None, (P_maps1, P_maps2, Q_maps1, Q_maps2), "rrrr")

    def gnl_con_sum(self, r_weights, R_maps):
        return _radial_sum("gnl_con_sum", r_weights, None, (R_maps,), "r")

    def gnl_con_disc_sum(self, r_weights, R_maps1, R_maps2):
        return _radial_sum("gnl_con_disc_sum", r_weights, None, (R_maps1, R_maps2), "rr")

    def gnl_dotdot_sum(self, rtau_weights, tau_arr, A_maps):
        return _radial_sum("gnl_dotdot_sum", rtau_weights, tau_arr, (A_maps,), "r")

    def gnl_dotdot_disc_sum(self, rtau_weights, tau_arr, A_maps1, A_maps2):
        return _radial_sum("gnl_dotdot_disc_sum", rtau_weights, tau_arr, (A_maps1, A_maps2), "rr")

    def gnl_dotdel_sum(self, rtau_weights, tau_arr, A_maps, B_maps, C_maps):
        return _radial_sum("gnl_dotdel_sum", rtau_weights, tau_arr, (A_maps, B_maps, C_maps), "rrc")

    def gnl_dotdel_disc_sum(self, rtau_weights, tau_arr, A_maps1, A_maps2, B_maps1, B_maps2, C_maps1, C_maps2):
        return _radial_sum("gnl_dotdel_disc_sum", rtau_weights, tau_arr,
                           (A_maps1, A_maps2, B_maps1, B_maps2, C_maps1, C_maps2), "rrrrcc")

    def gnl_deldel_sum(self, rtau_weights, B_maps, C_maps):
        return _radial_sum("gnl_deldel_sum", rtau_weights, None, (B_maps, C_maps), "rc")

    def gnl_deldel_disc_sum(self, rtau_weights, B1_maps, B2_maps, B3_maps, B4_maps, C1_maps, C2_maps, C3_maps,
                            C4_maps):
        return _radial_sum("gnl_deldel_disc_sum", rtau_weights, None,
                           (B1_maps, B2_maps, B3_maps, B4_maps, C1_maps, C2_maps, C3_maps, C4_maps), "rrrrcccc")


# -------------------------------------------------------------------- ideal_fisher.pyx mirrors
def r2c(re_arr, im_arr, nthreads=0):
    return _product("r2c", (re_arr, im_arr), "rr", True)


def r2cstar(re_arr, im_arr, nthreads=0):
    return _product("r2cstar", (re_arr, im_arr), "rr", True)


def multiplyRC(arrR, arrC, nthreads=0):
    return _product("multiplyRC", (arrR, arrC), "rc", True)


def multiplyRCstar(arrR, arrC, fac, nthreads=0):
    return _product("multiplyRCstar", (arrR, arrC), "rc", True, fac=fac)


def multiplyRC_sym(arrR, arrC, arrR2, arrC2, nthreads=0):
    return _product("multiplyRC_sym", (arrR, arrC, arrR2, arrC2), "rcrc", True)


def multiplyRCstar_sym(arrR, arrC, arrR2, arrC2, fac, nthreads=0):
    return _product("multiplyRCstar_sym", (arrR, arrC, arrR2, arrC2), "rcrc", True, fac=fac)


def multiplyRR(arr1, arr2, nthreads=0):
    return _product("multiplyRR", (arr1, arr2), "rr", False)


def multiplyRR_sym(arr1, arr2, arr1b, arr2b, nthreads=0):
    return _product("multiplyRR_sym", (arr1, arr2, arr1b, arr2b), "rrrr", False)


def compute_product_real_all(maps, F_maps, weights, pq_inds, F_inds, nthreads=0):
    """out = Sum_i weights[i] maps[pq_inds[i]] F_maps[F_inds[i]] for real [N_r, Npix] maps, one or two terms
    of equal weight: compute_productP_real_all / compute_productQ_real_all of ideal_fisher.pyx:177-190,
    :325-338 with the F maps real (their n1 = 0 form)."""
    w = [float(x) for x in weights]
    if len(w) == 1:
        return _product("product_real1", (maps[pq_inds[0]], F_maps[F_inds[0]]), "rr", False, fac=w[0])
    if len(w) == 2 and w[0] == w[1]:
        return _product("product_real2", (maps[pq_inds[0]], F_maps[F_inds[0]], maps[pq_inds[1]], F_maps[F_inds[1]]),
                        "rrrr", False, fac=w[0])
    raise ValueError("one term, or two terms of equal weight")


def compute_productP_real_all(P_map, F_PQ, weights, pq_inds, F_inds, nthreads=0):
    """ideal_fisher.pyx:177-190: Sum_i weights[i] P_map[pq_inds[i]] Re F_PQ[F_inds[i]] ([N_r, Npix] maps;
    one term, or two of equal weight, as the local-tauNL derivative uses)."""
    F = F_PQ.real if (isinstance(F_PQ, torch.Tensor) and F_PQ.is_complex()) or np.iscomplexobj(F_PQ) else F_PQ
    return compute_product_real_all(P_map, F, weights, pq_inds, F_inds)


def compute_productQ_real_all(Q_map, F_PQ, weights, pq_inds, F_inds, mu1_index, nthreads=0):
    """ideal_fisher.pyx:325-338: Sum_i weights[i] Q_map[pq_inds[i]] Re F_PQ[F_inds[i], mu1_index]."""
    F = F_PQ[:, mu1_index]
    F = F.real if (isinstance(F, torch.Tensor) and F.is_complex()) or np.iscomplexobj(F) else F
    return compute_product_real_all(Q_map, F, weights, pq_inds, F_inds)


def _i32(x):
    return torch.as_tensor(np.asarray(x, dtype=np.int32), device=_dev())


def compute_productPnmu_sym_all(Pnmu_maps, F_PQ, weights, n1, pq_inds, F_inds, nthreads=0):
    """ideal_fisher.pyx:195-212: Sum_i w_i [Re(P[pq_i, 0] F[F_i, 0]) + 2 Sum_{mu>=1} Re(P[pq_i, mu] F[F_i, mu])]
    for complex P [nP, n1+1, N_r, Npix] and F [nF, n1+1, N_r, Npix]; real [N_r, Npix]."""
    P, as_torch = _prep(Pnmu_maps, torch.complex128)
    F, _ = _prep(F_PQ, torch.complex128)
    ntot = P.shape[2] * P.shape[3]
    out = torch.empty(P.shape[2:], dtype=torch.float64, device=P.device)
    w = torch.as_tensor(np.asarray(weights, dtype=np.float64), device=P.device)
    pq, fi = _i32(pq_inds), _i32(F_inds)
    _lib.call("ps_product_pnmu_sym", ctypes.c_void_p(P.data_ptr()), ctypes.c_void_p(F.data_ptr()), int(n1), ntot,
              ctypes.c_void_p(w.data_ptr()), ctypes.c_void_p(pq.data_ptr()), ctypes.c_void_p(fi.data_ptr()), len(w),
              ctypes.c_void_p(out.data_ptr()), _stream())
    torch.cuda.current_stream().synchronize()  # the index arrays are released on return
    return _ret(out, as_torch)


def compute_productQ_complex_all(Q_map, F_PQ, weights, pq_inds, F_inds, mu1_index, nthreads=0):
    """ideal_fisher.pyx:343-357: Sum_i w_i Q[pq_i] F_PQ[F_i, mu1_index] (complex [N_r, Npix])."""
    Q, as_torch = _prep(Q_map, torch.float64)
    F, _ = _prep(F_PQ, torch.complex128)
    ntot = Q.shape[1] * Q.shape[2]
    out = torch.empty(Q.shape[1:], dtype=torch.complex128, device=Q.device)
    w = torch.as_tensor(np.asarray(weights, dtype=np.float64), device=Q.device)
    pq, fi = _i32(pq_inds), _i32(F_inds)
    _lib.call("ps_product_q_complex", ctypes.c_void_p(Q.data_ptr()), ctypes.c_void_p(F.data_ptr()), F.shape[1],
              int(mu1_index), ntot, ctypes.c_void_p(w.data_ptr()), ctypes.c_void_p(pq.data_ptr()),
              ctypes.c_void_p(fi.data_ptr()), len(w), ctypes.c_void_p(out.data_ptr()), _stream())
    torch.cuda.current_stream().synchronize()
    return _ret(out, as_torch)


def complex_to_complex(map1, map2, nthreads=0):
    """ideal_fisher.pyx:274-286: out[0] = map1^T + i map2^T, out[1] = map1^T - i map2^T ([2, n1, n0])."""
    a, as_torch = _prep(map1, torch.complex128)
    b, _ = _prep(map2, torch.complex128)
    out = torch.stack([(a + 1j * b).T, (a - 1j * b).T]).contiguous()
    return _ret(out, as_torch)


def r2cstar_inplace(re_arr, im_arr, out_arr, mu_index, nthreads=0):
    """ideal_fisher.pyx:42-47: out_arr[mu_index] = re - i im, in place."""
    v = r2cstar(re_arr, im_arr)
    if isinstance(out_arr, torch.Tensor):
        out_arr[mu_index] = torch.as_tensor(v, device=out_arr.device)
    else:
        out_arr[mu_index] = v.cpu().numpy() if isinstance(v, torch.Tensor) else v


def compute_productP_all(P_map, F_PQ, weights, pq_inds, F_inds, nthreads=0):
    """ideal_fisher.pyx:160-175: Sum_i w_i Re(P[pq_i] F_PQ[F_i]) for complex P (real [N_r, Npix])."""
    P, as_torch = _prep(P_map, torch.complex128)
    F, _ = _prep(F_PQ, torch.complex128)
    out = torch.zeros(P.shape[1:], dtype=torch.float64, device=P.device)
    for w, ip, iF in zip(np.asarray(weights, dtype=np.float64), pq_inds, F_inds):
        out += float(w) * (P[int(ip)] * F[int(iF)]).real
    return _ret(out, as_torch)


def compute_productPnmu_all(Pnmu_maps, conjPnmu_maps, F_PQ, weights, n1, pq_inds, F_inds, nthreads=0):
    """ideal_fisher.pyx:216-234: Sum_i w_i Re(P[pq_i, 0] F[F_i, n1] + Sum_{mu >= 1} (P[pq_i, mu] F[F_i, n1 + mu]
    + (-1)^(n1-mu) conj(Pc[pq_i, mu]) F[F_i, n1 - mu])) for the complex collider P^beta maps and those of conj(beta)."""
    P, as_torch = _prep(Pnmu_maps, torch.complex128)
    Pc, _ = _prep(conjPnmu_maps, torch.complex128)
    F, _ = _prep(F_PQ, torch.complex128)
    n1 = int(n1)
    out = torch.zeros(P.shape[2:], dtype=torch.float64, device=P.device)
    for w, ip, iF in zip(np.asarray(weights, dtype=np.float64), pq_inds, F_inds):
        ip, iF = int(ip), int(iF)
        acc = P[ip, 0] * F[iF, n1]
        for mu1 in range(1, n1 + 1):
            acc = acc + P[ip, mu1] * F[iF, n1 + mu1] + (-1.) ** (n1 - mu1) * Pc[ip, mu1].conj() * F[iF, n1 - mu1]
        out += float(w) * acc.real
    return _ret(out, as_torch)


def complex_to_complex_transpose(map1, map2, nthreads=0):
    """ideal_fisher.pyx:291-303: out[0] = map1 + i map2, out[1] = map1 - i map2 (no transpose)."""
    a, as_torch = _prep(map1, torch.complex128)
    b, _ = _prep(map2, torch.complex128)
    return _ret(torch.stack([a + 1j * b, a - 1j * b]).contiguous(), as_torch)


def integrate_pq_complex(flXs, P_FPQ_plus, P_FPQ_minus, ls, r_weights, out, inds, nthreads=0):
    """ideal_fisher.pyx:378-391: out[X, lm] += Sum_i 0.25 w_i (f[l, X, inds i] plus[lm, i] + conj(f) minus[lm, i])
    for complex f, as the two real radial sums of Re f (plus + minus) / 2 and Im f i (plus - minus) / 2."""
    f, _ = _prep(flXs, torch.complex128)
    pp, _ = _prep(P_FPQ_plus, torch.complex128)
    mm, _ = _prep(P_FPQ_minus, torch.complex128)
    integrate_pq(f.real.contiguous(), 0.5 * (pp + mm), ls, r_weights, out, inds)
    integrate_pq(f.imag.contiguous(), 0.5j * (pp - mm), ls, r_weights, out, inds)


def integrate_pq(flXs, P_FPQ, ls, r_weights, out, inds, nthreads=0):
    """ideal_fisher.pyx:361-375: out[X, lm] += Sum_i 0.5 w_i flXs[ls[lm], X, inds[i]] P_FPQ[lm, i], in place
    (out numpy or CUDA tensor), as one ps_radial_sum_lm launch."""
    inds = np.asarray(inds, dtype=np.int64)
    f, _ = _prep(np.asarray(flXs)[:, :, inds] if not isinstance(flXs, torch.Tensor) else flXs[:, :, inds],
                 torch.float64)
    m, _ = _prep(P_FPQ.T if isinstance(P_FPQ, torch.Tensor) else np.asarray(P_FPQ).T, torch.complex128)
    d_ls, _ = _prep(np.asarray(ls, dtype=np.int32), torch.int32)
    w = torch.as_tensor(0.5 * np.asarray(r_weights, dtype=np.float64)[:len(inds)], device=m.device)
    lsize, npol, nr = f.shape
    nlm = m.shape[1]
    res = torch.empty((npol, nlm), dtype=torch.complex128, device=m.device)
    _lib.call("ps_radial_sum_lm", ctypes.c_void_p(m.data_ptr()), 0, ctypes.c_void_p(w.data_ptr()),
              ctypes.c_void_p(f.data_ptr()), lsize, npol, nr, ctypes.c_void_p(d_ls.data_ptr()), nlm,
              ctypes.c_void_p(res.data_ptr()), _stream())
    if isinstance(out, torch.Tensor):
        out[:npol] += res.to(out.device)
    else:
        out[:npol] += res.cpu().numpy()


def tau_convolve_F(X, lm_L, F, r_weights, A=None, lm_w=None):
    """F_L convolution of harmonic maps X [N_r, nlm] (complex128, one lm list, CUDA):
    out[j, lm] = Sum_k F[L(lm), j, k] w_k X[k, lm] / sqrt(4 pi) with L = lm_L[lm] (int32, -1: out = 0),
    convolve_F_n000 of tauNL_utils.pyx:966-995 for F one n-slice [nL, N_r, N_r].  With A (and the m
    weights lm_w) it returns instead the scalar Sum_{lm, j} lm_w w_j Re(A[j, lm] conj(out[j, lm])),
    tau_sum_n0 (:604-647) of (A, X)."""
    X = X.contiguous()
    nr, nlm = X.shape
    lm_L = lm_L.to(torch.int32).contiguous()
    w = torch.as_tensor(np.asarray(r_weights, dtype=np.float64), device=X.device)
    if F.shape[1:] != (nr, nr) or lm_L.numel() != nlm or w.numel() != nr:
        raise ValueError("X, lm_L, F and r_weights do not match")
    nL = F.shape[0]
    if nlm and int(lm_L.max()) >= nL:
        raise ValueError("lm_L holds an L beyond F")
    FT = F.permute(1, 2, 0).contiguous()  # [j][k][L], the kernel's layout
    if A is None:
        out = torch.empty_like(X)
        _lib.call("ps_tau_convolve_F", ctypes.c_void_p(X.data_ptr()), None, ctypes.c_void_p(lm_L.data_ptr()), None,
                  ctypes.c_void_p(FT.data_ptr()), nL, ctypes.c_void_p(w.data_ptr()), nr, nlm,
                  ctypes.c_void_p(out.data_ptr()), None, None, 0, _stream())
        return out
    A = A.contiguous()
    lm_w = lm_w.to(torch.float64).contiguous()
    if A.shape != X.shape or lm_w.numel() != nlm:
        raise ValueError("A, lm_w do not match X")
    nb = ctypes.c_size_t()
    _lib.call("ps_tau_convolve_workspace_bytes", nlm, ctypes.byref(nb))
    ws = torch.empty(max(int(nb.value), 8), dtype=torch.uint8, device=X.device)
    dot = torch.zeros(1, dtype=torch.float64, device=X.device)
    _lib.call("ps_tau_convolve_F", ctypes.c_void_p(X.data_ptr()), ctypes.c_void_p(A.data_ptr()),
              ctypes.c_void_p(lm_L.data_ptr()), ctypes.c_void_p(lm_w.data_ptr()), ctypes.c_void_p(FT.data_ptr()), nL,
              ctypes.c_void_p(w.data_ptr()), nr, nlm, None, ctypes.c_void_p(dot.data_ptr()),
              ctypes.c_void_p(ws.data_ptr()), int(nb.value), _stream())
    return float(dot.item())


def lens_phi_sum(umap, vmap, nthreads=0):
    """Pixel sum of U and V maps of the lensing Phi estimator (ideal_fisher.pyx:124-139)."""
    npol, npix = np.shape(umap)[0], np.shape(umap)[1]
    return _product("lens_phi_sum", (umap, vmap), "cc", True, npol=npol, out_shape=(npix,))


def lens_phi_sum_sym(umap1, umap2, vmap1, vmap2, nthreads=0):
    """Symmetrised lensing Phi pixel sum (ideal_fisher.pyx:142-157)."""
    npol, npix = np.shape(umap1)[0], np.shape(umap1)[1]
    return _product("lens_phi_sum_sym", (umap1, umap2, vmap1, vmap2), "cccc", True, npol=npol, out_shape=(npix,))


def outer_product(Q4_a, Q4_b, nthreads=0, sym=False):
    """Fisher outer product of two [4, n_t, n_in] arrays (ideal_fisher.pyx:423-460)."""
    a, as_torch = _prep(Q4_a, torch.complex128)
    b, _ = _prep(Q4_b, torch.complex128)
    if a.dim() != 3 or b.dim() != 3 or a.shape[0] != 4 or b.shape[0] != 4 or a.shape[2] != b.shape[2]:
        raise ValueError("Q4 arrays must be [4, n_t, n_in] with equal n_in")
    na, nb, nin = a.shape[1], b.shape[1], a.shape[2]
    if sym:
        assert na == nb, "Matrix must be square!"
    fish = torch.empty((na, nb), dtype=torch.float64, device=a.device)
    if nin == 0:
        fish.zero_()
        return _ret(fish, as_torch)
    n = ctypes.c_size_t()
    _lib.call("ps_outer_product_workspace_bytes", na, nb, nin, ctypes.byref(n))
    ws = torch.empty(max(int(n.value), 8), dtype=torch.uint8, device=a.device)
    _lib.call("ps_outer_product", ctypes.c_void_p(a.data_ptr()), ctypes.c_void_p(b.data_ptr()), na, nb, nin,
              int(bool(sym)), ctypes.c_void_p(fish.data_ptr()), ctypes.c_void_p(ws.data_ptr()), int(n.value),
              _stream())
    return _ret(fish, as_torch)
