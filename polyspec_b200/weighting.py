"""S^-1 weighting on the GPU (mirror of polyspec/weighting.py).

``Weightings(base, mask, Cl_raw, noise_cov=None, inpainting_mask=None)``
builds the same quantities as the reference (polyspec/weighting.py:6-85):
the inverse noise covariance, the isotropic noise level ``Nl_iso``, the
signal covariance and its inverse per (l, m) and the harmonic preconditioner
``Sigmalm``; ``applySinv_ideal`` and ``applySinv_optimal`` keep their
signatures and return harmonic coefficients truncated at ``lmax``.

All arrays live on the GPU; the transforms are libpscuda SHTs.  numpy inputs
give numpy outputs; CUDA-tensor inputs give CUDA-tensor outputs.
``CGD`` is the reference's preconditioned conjugate-gradient solver
(polyspec/weighting.py:217-367) with vectors, dot products and the A and M
operators evaluated on the device.
"""
import ctypes
import os

import numpy as np
import torch

from . import _lib, healpix, lmops


def _per_lm(base, mat_l):
    """Per-l matrices [a, b, lmax+1] -> complex device tensor [a, b, nlm] (indexed by base.l_arr)."""
    t = torch.as_tensor(np.ascontiguousarray(mat_l), device=base.device)
    return t[..., base.dev('l_arr')].to(torch.complex128).contiguous()


class Weightings:
    def __init__(self, base, mask, Cl_raw, noise_cov=None, inpainting_mask=None):
        self.base = base
        self.mask = mask
        self.Cl_raw = Cl_raw
        self.pol = self.base.pol
        self.pixel_area = 4. * np.pi / (12 * self.base.Nside ** 2)
        nf = 1 + 2 * self.pol
        dev = base.device

        if noise_cov is not None:
            self.noise_cov = noise_cov
            self.noise_icov = np.zeros_like(self.noise_cov)
            self.noise_icov[self.noise_cov != 0] = 1. / self.noise_cov[self.noise_cov != 0]

        if inpainting_mask is not None:
            assert np.mean(inpainting_mask) == np.mean(inpainting_mask ** 2), "Inpainting mask should be a boolean array!"
            self.inpainting_mask = inpainting_mask
            if np.mean(1. * self.inpainting_mask) > 0.5:
                print("## %.2f%% of the pixels will be inpainted: is this mask correct?" % (np.mean(1. * self.inpainting_mask) * 100))
            if self.pol:
                assert len(self.inpainting_mask) == 3, "Must supply one mask for each polarization!"
            else:
                if len(self.inpainting_mask) != 1:
                    self.inpainting_mask = self.inpainting_mask.reshape(1, -1)

        self.beam_lm = self.base.beam_lm
        ls = np.arange(self.base.lmax + 1)

        if hasattr(self, 'noise_cov'):
            self.Nl_iso = np.zeros(nf)
            for i in range(nf):
                self.Nl_iso[i] = np.mean(self.noise_cov[i][np.asarray(self.mask)[i] > 0.99]) * self.pixel_area
            # per-l signal covariance and its inverse (polyspec/weighting.py:52-73)
            if self.pol:
                assert len(Cl_raw.keys()) == 6 or len(Cl_raw.keys()) == 4, \
                    "Must specify four or six input spectra: {ClTT, ClTE, ClEE, ClBB} or {ClTT, ClTE, ClTB, ClEE, ClEB, ClBB}"
                if len(Cl_raw.keys()) == 4:
                    Cl_raw['TB'] = Cl_raw['EB'] = 0. * Cl_raw['TT']
                C = np.asarray([[Cl_raw['TT'][ls], Cl_raw['TE'][ls], Cl_raw['TB'][ls]],
                                [Cl_raw['TE'][ls], Cl_raw['EE'][ls], Cl_raw['EB'][ls]],
                                [Cl_raw['TB'][ls], Cl_raw['EB'][ls], Cl_raw['BB'][ls]]])  # [3,3,l]
                Cl_l = np.moveaxis(C, 2, 0)  # [l,3,3]
                inv_l = np.zeros((3, 3, len(ls)))
                if np.sum(Cl_raw['BB']) == 0:
                    good_l = np.linalg.det(Cl_l[:, :2, :2]) > 0
                    inv_l[:2, :2, good_l] = np.moveaxis(np.linalg.inv(Cl_l[good_l, :2, :2]), 0, 2)
                else:
                    good_l = np.linalg.det(Cl_l) > 0
                    inv_l[:, :, good_l] = np.moveaxis(np.linalg.inv(Cl_l[good_l]), 0, 2)
            else:
                Cl_l = Cl_raw['TT'][ls].reshape(-1, 1, 1)
                good_l = Cl_l[:, 0, 0] > 0
                inv_l = np.zeros((1, 1, len(ls)))
                inv_l[:, :, good_l] = np.moveaxis(np.linalg.inv(Cl_l[good_l]), 0, 2)
            self.Cl_l_mat = Cl_l            # [l, a, b]
            self.inv_Cl_l_mat = inv_l       # [a, b, l]
            # harmonic preconditioner (polyspec/weighting.py:76-78), per l
            beam_l = self.base.beam[:, :len(ls)]
            inv_S = inv_l + np.einsum('il,jl,ij->ijl', beam_l, beam_l, np.diag(1. / self.Nl_iso))
            inv_S[:, :, :2] = inv_S[:, :, 2:3]
            self.Sigma_l = np.moveaxis(np.linalg.inv(np.moveaxis(inv_S, 2, 0)), 0, 2)  # [a, b, l]
            # device, per (l, m)
            self.d_inv_Cl = _per_lm(base, self.inv_Cl_l_mat)
            self.d_Sigma = _per_lm(base, self.Sigma_l)
            self.d_noise_cov = torch.as_tensor(np.asarray(self.noise_cov, dtype=np.float64).reshape(nf, -1), device=dev)
            self.d_noise_icov = torch.as_tensor(np.asarray(self.noise_icov, dtype=np.float64).reshape(nf, -1), device=dev)
            # x0 operator C B C_tot^-1 (polyspec/weighting.py:174), per l
            self.x0_l = np.einsum('lab,bl,bcl->acl', Cl_l, beam_l, self.base.inv_Cl_tot_mat[:, :, :len(ls)])
            self.d_x0op = _per_lm(base, self.x0_l)

        if not (type(mask) == float or type(mask) == int):
            if len(mask) == 1 or len(mask) == 3:
                assert len(mask[0]) == self.base.Npix, f'Mask has incorrect shape: {np.shape(mask)}'
            else:
                assert len(mask) == self.base.Npix, f'Mask has incorrect shape: {np.shape(mask)}'
        m = np.asarray(mask, dtype=np.float64)
        self.d_mask = torch.as_tensor(m.reshape(-1, self.base.Npix) if m.ndim else m, device=dev)
        if hasattr(self, 'noise_cov'):
            # W N^-1 W / A_pix  (the A_pix of to_lm cancels it: polyspec/weighting.py:277, :290)
            self.d_WNW = (self.d_mask ** 2 * self.d_noise_icov).contiguous()

    # ------------------------------------------------------------------
    def inpaint_map(self, input_map, n_average=50):
        """Linear inpainting (polyspec/weighting.py:87-146): per field, zero the inpainting
        region, then fill its zero pixels with the mean of their 8 neighbours pass by pass
        (each pass over the pixels still zero, all reading the previous pass) until none is
        left or a pass fills none, then smooth the region by n_average passes of the plain
        neighbour mean.  The averages are ``ps_inpaint_average`` over the GPU neighbour table
        of ``healpix.neighbours``; the pass bookkeeping (which pixels are still zero) is a
        device compaction."""
        assert hasattr(self, 'inpainting_mask'), "Must supply inpainting mask to use inpainting code!"
        x, as_torch = self.base._in(input_map, torch.float64)
        tmp = x.clone()
        if not hasattr(self, 'd_inpaint_filt'):
            self.d_inpaint_filt = torch.as_tensor(np.asarray(self.inpainting_mask) == 1, device=tmp.device)
        filt = self.d_inpaint_filt
        if int(filt.sum()) == 0:
            return self.base._out(tmp, as_torch)
        nb = healpix.neighbours(self.base.Nside, tmp.device)
        npix = tmp.shape[-1]
        st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

        def average(src, pix, weighted, dst):  # pix: int32 list held by the caller
            _lib.call("ps_inpaint_average", ctypes.c_void_p(src.data_ptr()), ctypes.c_void_p(pix.data_ptr()),
                      pix.numel(), ctypes.c_void_p(nb.data_ptr()), npix, int(weighted),
                      ctypes.c_void_p(dst.data_ptr()), st)

        for field in range(1 + 2 * self.pol):
            this = tmp[field].clone()
            if float(torch.sum(this)) == 0:
                continue
            fm = filt[field]
            this[fm] = 0
            inpaint_pix = torch.nonzero((tmp[field] == 0) & fm).flatten().to(torch.int32)
            while True:
                nxt = this.clone()
                average(this, inpaint_pix, True, nxt)
                this = nxt
                next_inpaint = torch.nonzero((this == 0) & fm).flatten().to(torch.int32)
                if next_inpaint.numel() == 0:
                    break
                if next_inpaint.numel() == inpaint_pix.numel():
                    print("# Inpainting field %d failed!" % field)
                    break
                inpaint_pix = next_inpaint
            pix = torch.nonzero(fm).flatten().to(torch.int32)
            other = this.clone()
            for _ in range(n_average):
                average(this, pix, False, other)
                this, other = other, this
            tmp[field] = this
        return self.base._out(tmp, as_torch)

    def applySinv_optimal(self, input_map, preconditioner='pseudo_inverse', nstep=25, thresh=1e-4, verb=False,
                          input_type='map', lmax=None):
        """Optimal S^-1 by preconditioned CG from the ideal (Wiener) start
        (polyspec/weighting.py:148-184).  Output in harmonic space, l <= lmax."""
        assert input_type == 'map', "Optimal weighting should be applied only to pixel-space data!"
        if not hasattr(self, 'noise_cov'):
            raise Exception("The CGD solver requires a pixel-space noise covariance")
        if lmax is None:
            lmax = self.base.lmax
        d, as_torch = self.base._in(input_map, torch.float64)
        if hasattr(self, 'inpainting_mask'):
            d = self.inpaint_map(d)
        if preconditioner in ('learned', 'cut'):
            return self.base._out(self.batched_applySinv_optimal(d[None], preconditioner=preconditioner,
                                                                 nstep=nstep, thresh=thresh, verb=verb,
                                                                 lmax=lmax, _inpainted=True)[0], as_torch)
        x0 = torch.einsum('abi,bi->ai', self.d_x0op, self.base.to_lm(d))
        cgd = CGD(self, d, x0=x0, preconditioner=preconditioner, verb=verb)
        cgd.run(nstep=nstep, thresh=thresh)
        self.last_cgd = cgd
        lfilt = torch.as_tensor(self.base.l_arr <= lmax, device=self.base.device)
        return self.base._out(cgd.get_ivar_lm()[:, lfilt], as_torch)

    def batched_applySinv_optimal(self, maps, preconditioner='harmonic', nstep=25, thresh=1e-4, verb=False,
                                  lmax=None, _inpainted=False):
        """applySinv_optimal for a batch of maps [B, nfield, Npix] (CUDA tensor), solved
        as B lockstep CGs with batched SHTs; returns [B, nfield, nlm(lmax)]."""
        if lmax is None:
            lmax = self.base.lmax
        d = maps.to(device=self.base.device, dtype=torch.float64)
        if hasattr(self, 'inpainting_mask') and not _inpainted:
            d = torch.stack([self.inpaint_map(m) for m in d])
        lm = self.base.to_lm_batch(d)
        x0 = lmops.matvec3(self.real3('x0op'), lm) if self.pol else torch.einsum('abi,nbi->nai', self.d_x0op, lm)
        # the learned CG hands a system to the plain CG after half the step budget
        cgd = BatchedCGD(self, d, x0, preconditioner=preconditioner, learned_max_steps=max(1, nstep // 2))
        cgd.run(nstep=nstep, thresh=thresh, verb=verb)
        self.last_cgd = cgd
        lfilt = torch.as_tensor(self.base.l_arr <= lmax, device=self.base.device)
        return cgd.get_ivar_lm()[:, :, lfilt]

    def real3(self, name):
        """Float64 copy of the per-(l, m) 3x3 'Sigma', 'inv_Cl' or 'x0op' for the vector kernels."""
        cache = self.__dict__.setdefault('_real3', {})
        if name not in cache:
            cache[name] = lmops.real3({'Sigma': self.d_Sigma, 'inv_Cl': self.d_inv_Cl, 'x0op': self.d_x0op}[name])
        return cache[name]

    def roundtrip_operands(self):
        """(pixel weight W N^-1 W / A_pix [nf, npix], beam [nf, nlm]) as float64 device arrays for the
        fused CG operator, or None (FP64 plans, no noise covariance, or PS_FUSED_A=0)."""
        if self.base.prec == 'fp64' or not hasattr(self, 'd_WNW') or os.environ.get("PS_FUSED_A", "1") == "0":
            return None
        if getattr(self, '_rt_ops', None) is None:
            w = (self.d_WNW / self.pixel_area).expand(1 + 2 * self.pol, -1).contiguous()
            beam = self.base.dev('beam_lm').real.to(torch.float64).contiguous()
            self._rt_ops = (w, beam)
        return self._rt_ops

    def cut_preconditioner(self):
        """The masked-band preconditioner of this Weightings (built on first use)."""
        if getattr(self, '_cut', None) is None:
            from .cutprec import CutPreconditioner
            self._cut = CutPreconditioner(self)
        return self._cut

    def make_applySinv(self, kind='optimal', **kw):
        """A callable with the reference applySinv signature and a ``.batched``
        method (used by PSpecBin.compute_fisher_contribution(batched=True))."""
        W = self

        class _ApplySinv:
            def __call__(self, x, input_type='map', lmax=None):
                if kind == 'ideal':
                    return W.applySinv_ideal(x, input_type=input_type, lmax=lmax)
                return W.applySinv_optimal(x, input_type=input_type, lmax=lmax, **kw)

            def batched(self, maps, lmax=None):
                if kind == 'ideal':
                    return W.batched_applySinv_ideal(maps, lmax=lmax)
                return W.batched_applySinv_optimal(maps, lmax=lmax, **kw)

        return _ApplySinv()

    def batched_applySinv_ideal(self, maps, lmax=None):
        """applySinv_ideal on a leading batch axis: maps [B, nfield, Npix] (CUDA) ->
        [B, nfield, nlm(lmax)], one batched adjoint transform per spin."""
        if lmax is None:
            lmax = self.base.lmax
        if hasattr(self, 'inpainting_mask'):
            maps = torch.stack([self.inpaint_map(m) for m in maps])
        lfilt = torch.as_tensor(self.base.l_arr <= lmax, device=self.base.device)
        icov = self.base.dev('inv_Cl_tot_lm_mat')
        beam = self.base.dev('beam_lm')
        lm = self.base.to_lm_batch(maps)
        return beam[:, lfilt] * torch.einsum("abl,nbl->nal", icov[:, :, lfilt], lm[:, :, lfilt])

    def applySinv_ideal(self, input_map, input_type='map', lmax=None):
        """Ideal S^-1 = beam C_tot^-1 Y^dagger W (polyspec/weighting.py:186-214)."""
        if lmax is None:
            lmax = self.base.lmax
        lfilt = torch.as_tensor(self.base.l_arr <= lmax, device=self.base.device)
        icov = self.base.dev('inv_Cl_tot_lm_mat')
        beam = self.base.dev('beam_lm')
        if input_type == 'harmonic':
            assert np.mean(self.mask) == 1, "Harmonic-space S^-1 requires a unit mask!"
            x, as_torch = self.base._in(input_map, torch.complex128)
            out = beam[:, lfilt] * torch.einsum("abl,bl->al", icov[:, :, lfilt], x)
            return self.base._out(out, as_torch)
        x, as_torch = self.base._in(input_map, torch.float64)
        if hasattr(self, 'inpainting_mask'):
            x = self.inpaint_map(x)
        input_lm = self.base.to_lm(x)
        out = beam[:, lfilt] * torch.einsum("abl,bl->al", icov[:, :, lfilt], input_lm[:, lfilt])
        return self.base._out(out, as_torch)


class BatchedCGD:
    """B independent copies of the reference CG (polyspec/weighting.py:217-367): vectors
    are [B, nfield, nlm] and each right-hand side keeps its own alpha, beta and stopping
    test (err_b = rz_b / rz0_b < thresh freezes system b, as a separate run would stop).
    r and p hold only the systems still running (rows dropped once, when a system
    stops), and A and M apply to them as one batched SHT pair, so the work is the sum
    of the separate runs' work, not B times the slowest run's.  The vector updates are
    fused kernels (x += alpha p with r -= alpha Ap, p = z + beta p, C^-1 p added to the
    round trip in place, r^T Sigma r without storing Sigma r)."""

    def __init__(self, weightings, d, x0, preconditioner='harmonic', learned_max_steps=None):
        self.base = weightings.base
        self.W = weightings
        self.preconditioner = preconditioner
        self.w = self.base.dev('m_weight')
        if preconditioner == 'learned':
            # learned band preconditioner (polyspec_b200.learned); the convergence statistic
            # is the plain CG's r^T Sigma r / b^T Sigma b, and a system that misbehaves or
            # exceeds learned_max_steps continues with the plain harmonic CG
            self.learned = getattr(weightings, 'learned', None)
            if self.learned is None or self.learned.L is None:
                raise Exception("preconditioner='learned' needs a trained Weightings.learned")
            self.learned_max_steps = learned_max_steps
        elif preconditioner == 'cut':
            # masked-band preconditioner (polyspec_b200.cutprec), stopped like 'learned'
            self.cut = weightings.cut_preconditioner()
        b0 = self._get_b(d)
        self.x0 = x0
        b = b0 - self._apply_A(x0)
        self.x = torch.zeros_like(b)
        self.r = b.clone()
        B = b.shape[0]
        self.use_learned = torch.full((B,), preconditioner == 'learned', dtype=torch.bool, device=b.device)
        z = self._apply_M(self.r, self.use_learned)
        self.rz = self.dot(self.r, z)
        if preconditioner in ('learned', 'cut'):
            # the stopping test uses Sigma whatever M is (no M b0 needed)
            self.stat0 = self._quad_sigma(b0)
            self.rz0 = self.stat0
        else:
            self.rz0 = self.dot(b0, self._apply_M(b0, self.use_learned))
        self.p = z
        # rows of r and p: the systems still running (slots = their indices); x stays full-size
        self.slots = torch.arange(B, device=b.device)
        self.i = 0
        self.iters = torch.zeros(B, dtype=torch.int64, device=b.device)
        self.active = torch.ones(B, dtype=torch.bool, device=b.device)
        self.err = self._stop_stat(self.r, self.rz, self.use_learned, torch.arange(B, device=b.device))

    def _pol(self, x):
        return x.dim() == 3 and x.shape[1] == 3

    def _sigma(self, ilm):
        if self._pol(ilm):
            return lmops.matvec3(self.W.real3('Sigma'), ilm)
        return torch.einsum('abi,nbi->nai', self.W.d_Sigma, ilm)

    def _stop_stat(self, r, rz, learned_mask, idx):
        """Stopping statistic: rz/rz0 of the plain CG (= r^T Sigma r / b^T Sigma b)."""
        if self.preconditioner not in ('learned', 'cut'):
            return rz / self.rz0[idx]
        return self._quad_sigma(r) / self.stat0[idx]

    def _quad_sigma(self, r):
        """r^T Sigma r per system (m-weighted; Sigma r not stored for T, E, B)."""
        if self._pol(r):
            return lmops.quad_dot(self.W.real3('Sigma'), r, self.w)
        return self.dot(r, self._sigma(r))

    def dot(self, a, b):
        if self._pol(a):
            return lmops.dot(a, b, self.w)
        return torch.sum((a * b.conj()).real * self.w, dim=(-2, -1))

    def _get_b(self, d):
        m = d * self.W.d_noise_icov / self.W.pixel_area
        return self.base.to_lm_batch(m * self.W.d_mask) * self.base.dev('beam_lm')

    def _apply_Cinv(self, ilm):
        if self._pol(ilm):
            return lmops.matvec3(self.W.real3('inv_Cl'), ilm)
        return torch.einsum('abi,nbi->nai', self.W.d_inv_Cl, ilm)

    def _apply_A(self, ilm):
        # mixed plans with Legendre tables: B Y^H (W N^-1 W / A_pix) Y B in one fused call per spin
        # (ps_sht_weighted_roundtrip; the maps stay in shared memory)
        rt = self.W.roundtrip_operands()
        if rt is not None:
            out = self.base.plan().weighted_roundtrip(ilm, rt[0], rt[1], np.pi / (3. * self.base.Nside ** 2))
            if out is not None:
                B, nf = ilm.shape[0], ilm.shape[1]
                self.base.n_SHTs_reverse += B * (1 + (nf == 3))
                self.base.n_SHTs_forward += B * (1 + (nf == 3))
                return self._add_Cinv(ilm, out)
        beam = self.base.dev('beam_lm')
        m = self.base.to_map_batch(ilm * beam)
        m = m * (self.W.d_WNW / self.W.pixel_area)
        y = self.base.to_lm_batch(m)
        y *= beam
        return self._add_Cinv(ilm, y)

    def _add_Cinv(self, ilm, y):
        """y + C^-1 ilm (in place on y for T, E, B)."""
        if self._pol(ilm) and y.is_contiguous():
            return lmops.matvec3_add(self.W.real3('inv_Cl'), ilm, y)
        return self._apply_Cinv(ilm) + y

    def _fallback_M(self, r):
        """Preconditioner of a system the learned CG hands back: the learned operator's own base
        (the masked-band preconditioner when it sits on that one, else the harmonic Sigma)."""
        cut = getattr(self.learned, 'cut', None) if hasattr(self, 'learned') else None
        return cut.apply(r) if cut is not None else self._sigma(r)

    def _apply_M(self, ilm, learned_mask=None):
        Sig = self.W.d_Sigma
        if self.preconditioner == 'cut':
            return self.cut.apply(ilm)
        if self.preconditioner == 'learned':
            z = self.learned.apply(ilm)
            if learned_mask is not None and not bool(learned_mask.all()):
                plain = ~learned_mask
                z[plain] = self._fallback_M(ilm[plain])
            return z
        if self.preconditioner == 'harmonic':
            return self._sigma(ilm)
        elif self.preconditioner == 'pseudo_inverse':
            beam = self.base.dev('beam_lm')
            Nl = torch.as_tensor(self.W.Nl_iso, device=self.base.device)[:, None]
            alm = torch.einsum('abi,nbi->nai', Sig, ilm)
            alm_signal = self._apply_Cinv(alm)
            alm_noise = alm * beam / Nl
            alm_noise = self.base.to_lm_batch(self.W.d_noise_cov * self.base.to_map_batch(alm_noise)) * self.W.pixel_area
            alm_noise = alm_noise * beam / Nl
            return torch.einsum('abi,nbi->nai', Sig, alm_noise + alm_signal)
        raise Exception("Unknown preconditioner %s specified!" % self.preconditioner)

    def step(self):
        keep = self.active[self.slots]
        if not bool(keep.all()):
            # systems stopped since the last step: drop their rows (once, not every step)
            self.r = self.r[keep]
            self.p = self.p[keep]
            self.slots = self.slots[keep]
        idx = self.slots
        if idx.numel() == 0:
            return
        p, r = self.p, self.r
        rz = self.rz[idx]
        lm = self.use_learned[idx]
        Ap = self._apply_A(p)
        alpha = rz / self.dot(p, Ap)
        fused = r.is_contiguous() and p.is_contiguous() and Ap.is_contiguous() and self.x.is_contiguous()
        if fused:
            lmops.xr_update(self.x, idx, alpha, p, r, Ap)  # x[idx] += alpha p, r -= alpha Ap
        else:
            self.x[idx] = self.x[idx] + alpha[:, None, None] * p
            r = r - alpha[:, None, None] * Ap
        z = self._apply_M(r, lm)
        next_rz = self.dot(r, z)
        beta = next_rz / rz
        if fused and z.is_contiguous():
            lmops.direction(p, z, beta)  # p = z + beta p
        else:
            p = z + beta[:, None, None] * p
        if self.preconditioner == 'learned':
            # fallback: a learned system whose r^T M r is not positive and finite, or that
            # has used its learned step budget, restarts as plain harmonic CG from x
            bad = lm & ~(torch.isfinite(next_rz) & (next_rz > 0))
            if self.learned_max_steps is not None:
                bad |= lm & (self.iters[idx] + 1 >= self.learned_max_steps)
            if bool(bad.any()):
                zs = self._fallback_M(r[bad])
                p[bad] = zs
                next_rz[bad] = self.dot(r[bad], zs)
                lm = lm & ~bad
                self.use_learned[idx] = lm
        self.r, self.p = r, p
        self.err[idx] = self._stop_stat(r, next_rz, lm, idx)
        self.rz[idx] = next_rz
        self.iters[idx] += 1
        self.i += 1

    def run(self, nstep=10, thresh=1e-6, verb=False):
        for i in range(nstep):
            self.step()
            self.active &= ~(self.err < thresh)
            if verb:
                print("batched CGD step %d: max error = %.2e, active %d" % (self.i, float(self.err.max()),
                                                                             int(self.active.sum())))
            if not bool(self.active.any()):
                break
        if bool(self.active.any()):
            print("CGD did not converge to %.2e threshold after %d steps. Final error = %.2e"
                  % (thresh, nstep, float(self.err.max())))

    def get_ivar_lm(self):
        return self._apply_Cinv(self.x + self.x0)


class CGD:
    """Preconditioned CG for A x = b, A = C^-1 + P^dagger N^-1 P, P = W Y B
    (polyspec/weighting.py:217-367), on device tensors."""

    def __init__(self, weightings, d, x0=[], test_b=[], preconditioner='pseudo_inverse', verb=False):
        self.preconditioner = preconditioner
        self.base = weightings.base
        self.weightings = weightings
        self.verb = verb
        if len(test_b) == 0:
            b0 = self._get_b(d.clone())
        else:
            print("Running in test mode!")
            assert len(d) == 0, "Cannot specify both d and test_b!"
            b0, _ = self.base._in(test_b, torch.complex128)
            b0 = b0.clone()
        if len(x0) != 0:
            self.x0 = x0
            b = b0 - self._apply_A(self.x0)
        else:
            self.x0 = 0.
            b = b0
        self.x = torch.zeros_like(b)
        self.r = b.clone()
        self.w = self.base.dev('m_weight')
        z = self._apply_M(self.r)
        self.rz = self.dot(self.r, z)
        self.rz0 = float(self.dot(b0, self._apply_M(b0)))
        self.p = z
        self.i = 0
        self.err = self.rz / self.rz0

    def dot(self, a, b):
        """m-weighted real inner product sum a b^* (1 + [m > 0]) (polyspec/weighting.py:255)."""
        return float(torch.sum((a * b.conj()).real * self.w))

    # filtering
    def _apply_beam(self, ilm):
        return ilm * self.base.dev('beam_lm')

    def _apply_mask(self, imap):
        return imap * self.weightings.d_mask

    def _apply_Ninv(self, imap):
        return imap * self.weightings.d_noise_icov / self.weightings.pixel_area

    def _apply_Cinv(self, ilm):
        return torch.einsum('abi,bi->ai', self.weightings.d_inv_Cl, ilm)

    def _pointing(self, ilm):
        return self._apply_mask(self.base.to_map(self._apply_beam(ilm)))

    def _pointing_adjoint(self, imap):
        return self._apply_beam(self.base.to_lm(self._apply_mask(imap)))

    def _get_b(self, d):
        return self._pointing_adjoint(self._apply_Ninv(d))

    def _apply_A(self, ilm):
        # C^-1 p + B Y^dagger W N^-1 W Y B p; W and N^-1 fused into one pixel weight
        m = self.base.to_map(self._apply_beam(ilm))
        m = m * (self.weightings.d_WNW / self.weightings.pixel_area)
        return self._apply_Cinv(ilm) + self._apply_beam(self.base.to_lm(m))

    def _apply_M(self, ilm):
        Sig = self.weightings.d_Sigma
        if self.preconditioner == 'harmonic':
            return torch.einsum('abi,bi->ai', Sig, ilm)
        elif self.preconditioner == 'pseudo_inverse':
            W = self.weightings
            alm = torch.einsum('abi,bi->ai', Sig, ilm)
            alm_signal = torch.einsum('abi,bi->ai', W.d_inv_Cl, alm)
            Nl = torch.as_tensor(W.Nl_iso, device=self.base.device)[:, None]
            alm_noise = alm * self.base.dev('beam_lm') / Nl
            alm_noise = self.base.to_lm(W.d_noise_cov * self.base.to_map(alm_noise)) * W.pixel_area
            alm_noise = alm_noise * self.base.dev('beam_lm') / Nl
            return torch.einsum('abi,bi->ai', Sig, alm_noise + alm_signal)
        else:
            raise Exception("Unknown preconditioner %s specified!" % self.preconditioner)

    def step(self):
        Ap = self._apply_A(self.p)
        alpha = self.rz / self.dot(self.p, Ap)
        self.x += alpha * self.p
        self.r -= alpha * Ap
        del Ap
        z = self._apply_M(self.r)
        next_rz = self.dot(self.r, z)
        self.err = next_rz / self.rz0
        beta = next_rz / self.rz
        self.rz = next_rz
        self.p = z + beta * self.p
        self.i += 1

    def run(self, nstep=10, thresh=1e-6):
        for i in range(nstep):
            self.step()
            if self.verb:
                print("CGD step %d: error = %.2e" % (self.i, self.err))
            if self.err < thresh:
                if self.verb:
                    print("CGD terminating at step %d" % self.i)
                break
        if i == nstep - 1 and self.err > thresh:
            print("CGD did not converge to %.2e threshold after %d steps. Final error = %.2e" % (thresh, nstep, self.err))

    def get_wiener_lm(self):
        return self.x + self.x0

    def get_wiener_map(self):
        return self.base.to_map(self.x + self.x0)

    def get_ivar_lm(self):
        return self._apply_Cinv(self.x + self.x0)

    def get_ivar_map(self):
        return self.base.to_map(self._apply_Cinv(self.x + self.x0))
