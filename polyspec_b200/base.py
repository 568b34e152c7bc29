"""PolySpec base class with the CUDA backend (mirror of polyspec/base.py).

``PolySpec(Nside, Cl_tot, beam=[], pol=True, backend='cuda', nthreads=0)``
keeps the reference constructor (polyspec/base.py:20) and every SHT wrapper
signature (``to_lm``, ``to_map``, ``to_lm_vec``, ``to_map_vec``,
``to_lm_spin``, ``to_map_spin``, ``compute_spin_transform_map``,
``generate_data``, ``applyAinv``), the attributes the estimators read
(``l_arr, m_arr, m_weight, inv_Cl_tot_lm_mat, beam_lm, A_pix, lmax, ...``),
the asserts on shapes and the counters ``n_SHTs_forward/reverse`` and
``time_sht`` (polyspec/base.py:113-127).

Every transform runs on the GPU through libpscuda.  Wrappers accept numpy
arrays (returning numpy, as the reference does) or CUDA tensors (returning
CUDA tensors, so estimator pipelines stay on the device).  There is no CPU
fallback: constructing the class without a GPU or without the built library
raises.

Extensions beyond the reference (optional keywords): ``lmax=`` fixes the
harmonic band limit used by default (the reference hard-codes 3 Nside - 1,
polyspec/base.py:30); ``prec='mixed'`` runs the SHTs on the mixed-precision
path (tensor-core Legendre synthesis, FP32 contractions and ring FFTs, FP64
inputs and outputs) instead of the FP64 path; with ``autotune=True`` (default)
each transform size runs whichever of the two pipelines measured faster on its
first call (the FP64 one for a few maps, the mixed one for batches).
"""
import os
import time

import numpy as np
import torch

from .sht import SHTPlan, nalm as _nalm


def getlm(lmax):
    """(l, m) of every coefficient in the HEALPix m-major order (healpy.Alm.getlm)."""
    m = np.concatenate([np.full(lmax + 1 - mm, mm, dtype=np.int64) for mm in range(lmax + 1)])
    l = np.concatenate([np.arange(mm, lmax + 1, dtype=np.int64) for mm in range(lmax + 1)])
    return l, m


def synalm_numpy(cls_rows, lmax, nfield):
    """Gaussian alm with covariance C_l, drawn from numpy's global generator.

    ``cls_rows`` follows healpy's ``new=False`` order: rows of the upper
    triangle (TT, TE, TB, EE, EB, BB) for three fields, (TT,) for one.
    Draw order: one ``standard_normal((nfield, nalm, 2))`` call; for m > 0 the
    pair gives (re + i im)/sqrt(2), for m = 0 the first number is used.  The
    field correlation is applied with the symmetric square root of C_l.
    """
    l, m = getlm(lmax)
    n = len(l)
    z = np.random.standard_normal((nfield, n, 2))
    zc = np.where(m[None] > 0, (z[..., 0] + 1j * z[..., 1]) / np.sqrt(2.0), z[..., 0] + 0j)
    C = np.zeros((lmax + 1, nfield, nfield))
    k = 0
    for i in range(nfield):
        for j in range(i, nfield):
            C[:, i, j] = C[:, j, i] = np.asarray(cls_rows[k])[:lmax + 1]
            k += 1
    w, V = np.linalg.eigh(C)
    S = np.einsum("lij,lj,lkj->lik", V, np.sqrt(np.clip(w, 0.0, None)), V)
    return np.einsum("nij,jn->in", S[l], zc)


class PolySpec:
    """Base class of PolySpec on one B200 (see module docstring)."""

    def __init__(self, Nside, Cl_tot, beam=[], pol=True, backend="cuda", nthreads=0, lmax=None, device=None,
                 prec="fp64", autotune=True):
        if backend != "cuda":
            raise Exception("polyspec_b200 implements the 'cuda' backend only")
        if not torch.cuda.is_available():
            raise RuntimeError("the 'cuda' backend needs a CUDA GPU")
        self.Nside = Nside
        self.pol = pol
        self.backend = backend
        if prec not in ("fp64", "mixed"):
            raise ValueError("prec must be 'fp64' or 'mixed'")
        self.prec = prec
        self.autotune = autotune
        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)

        self.Npix = 12 * Nside ** 2
        self.A_pix = 4. * np.pi / self.Npix
        self.lmax = 3 * self.Nside - 1 if lmax is None else int(lmax)
        self.l_arr, self.m_arr = getlm(self.lmax)
        if nthreads <= 0:
            self.nthreads = len(os.sched_getaffinity(0))
        else:
            self.nthreads = nthreads

        self.indices = {'T': 0, 'E': 1, 'B': 2}
        self.parities = {'T': 1, 'E': 1, 'B': -1}

        ls = np.arange(self.lmax + 1)
        if self.pol:
            assert len(Cl_tot.keys()) == 6 or len(Cl_tot.keys()) == 4, \
                "Must specify four or six input spectra: {ClTT, ClTE, ClEE, ClBB} or {ClTT, ClTE, ClTB, ClEE, ClEB, ClBB}"
            if len(Cl_tot.keys()) == 4:
                Cl_tot['TB'] = Cl_tot['EB'] = 0. * Cl_tot['TT']
        for k in Cl_tot.keys():
            assert len(Cl_tot[k]) >= len(ls), "Cl_tot must contain every ell mode from l=0 to l=lmax!"
        self.Cl_tot = Cl_tot.copy()

        if len(beam) == 0:
            self.beam = np.asarray([1. + 0. * self.Cl_tot['TT'] for _ in range(1 + 2 * self.pol)])
        else:
            if self.pol:
                assert len(beam) == 2 or len(beam) == 3, "Beam must contain temperature and polarization or T/E/B components"
                if len(beam) == 2:
                    self.beam = np.asarray([beam[0].copy(), beam[1].copy(), beam[1].copy()])
                else:
                    self.beam = np.asarray([beam[0].copy(), beam[1].copy(), beam[2].copy()])
            else:
                assert (len(beam) == 1 or len(beam) == len(Cl_tot['TT'])), "Beam must contain the same ells as Cl_tot"
                self.beam = np.asarray(beam).copy().reshape(1, -1)
        for i in range(len(self.beam)):
            assert len(self.beam[i]) >= len(ls), "Beam must contain every ell mode from l=0 to l=lmax!"

        self.m_weight = (1. + 1. * (self.m_arr > 0.))

        # the spin +-1/2 recombinations (numpy forms of polyspec/base.py:87-89)
        self.to_plus_minus = lambda map: _to_plus_minus(map)
        self.to_plus_minus_complex = lambda map, spin: _to_plus_minus_complex(map, spin)
        self.to_real_imag = lambda mapP, mapM: _to_real_imag(mapP, mapM)

        if pol:
            Cl_tot_mat = np.moveaxis(np.asarray([[self.Cl_tot['TT'], self.Cl_tot['TE'], self.Cl_tot['TB']],
                                                 [self.Cl_tot['TE'], self.Cl_tot['EE'], self.Cl_tot['EB']],
                                                 [self.Cl_tot['TB'], self.Cl_tot['EB'], self.Cl_tot['BB']]]), [2, 1, 0], [0, 2, 1])
            Cl_tot_mat = Cl_tot_mat[:len(ls)]
            good_l = np.linalg.det(Cl_tot_mat) > 0
            self.inv_Cl_tot_mat = np.zeros((3, 3, len(ls)), dtype=np.float64, order='C')
            self.inv_Cl_tot_mat[:, :, good_l] = np.moveaxis(np.linalg.inv(Cl_tot_mat[good_l]), [0, 1, 2], [2, 1, 0])
        else:
            good_l = self.Cl_tot['TT'][:len(ls)] > 0
            self.inv_Cl_tot_mat = np.zeros((1, 1, len(ls)), dtype=np.float64, order='C')
            self.inv_Cl_tot_mat[:, :, good_l] = 1. / self.Cl_tot['TT'][None, None, :len(ls)][:, :, good_l]

        self.inv_Cl_tot_lm_mat = np.asarray(self.inv_Cl_tot_mat[:, :, self.l_arr], order='C')
        self.beam_lm = np.asarray(self.beam[:, self.l_arr], order='C')

        self.n_SHTs_forward = 0
        self.n_SHTs_reverse = 0
        self.time_sht = 0.

        self._plans = {}
        self._dev_cache = {}

    # ------------------------------------------------------------------ device helpers
    def plan(self, lmax=None):
        lmax = self.lmax if lmax is None else int(lmax)
        p = self._plans.get(lmax)
        if p is None:
            p = SHTPlan(self.Nside, lmax, device=self.device, prec=self.prec, autotune=self.autotune)
            self._plans[lmax] = p
        return p

    def dev(self, name, lmax=None):
        """Device copy (torch) of a per-(l,m) table restricted to l <= lmax."""
        lmax = self.lmax if lmax is None else int(lmax)
        key = (name, lmax)
        t = self._dev_cache.get(key)
        if t is None:
            filt = self.l_arr <= lmax
            if name == 'beam_lm':
                arr = self.beam_lm[:, filt]
            elif name == 'inv_Cl_tot_lm_mat':
                arr = self.inv_Cl_tot_lm_mat[:, :, filt].astype(np.complex128)
            elif name == 'm_weight':
                arr = self.m_weight[filt]
            elif name == 'l_arr':
                arr = self.l_arr[filt]
            else:
                raise KeyError(name)
            t = torch.as_tensor(np.ascontiguousarray(arr), device=self.device)
            self._dev_cache[key] = t
        return t

    def _in(self, x, dtype):
        if isinstance(x, torch.Tensor):
            return x.to(device=self.device, dtype=dtype), True
        return torch.as_tensor(np.asarray(x), dtype=dtype, device=self.device), False

    @staticmethod
    def _out(t, as_torch):
        return t if as_torch else t.cpu().numpy()

    def timer_func(func):
        def wrap_func(self, *args, **kwargs):
            t1 = time.time()
            result = func(self, *args, **kwargs)
            t2 = time.time()
            self.time_sht += t2 - t1
            return result
        return wrap_func

    # ------------------------------------------------------------------ batched device transforms
    def to_map_batch(self, alm, lmax=None):
        """alm [B, nfield, nlm] (T or T,E,B) -> maps [B, nfield, Npix] (T or T,Q,U), one
        batched libpscuda call per spin; counts like B calls of to_map."""
        lmax = self.lmax if lmax is None else int(lmax)
        P = self.plan(lmax)
        B, nf = alm.shape[0], alm.shape[1]
        self.n_SHTs_reverse += B * (1 + (nf == 3))
        out = torch.empty((B, nf, self.Npix), dtype=torch.float64, device=self.device)
        out[:, 0] = P.synthesis(alm[:, 0].contiguous(), 0)
        if nf == 3:
            out[:, 1:] = P.synthesis(alm[:, 1:].contiguous(), 2)
        return out

    def to_lm_batch(self, maps, lmax=None):
        """maps [B, nfield, Npix] -> alm [B, nfield, nlm], scaled as to_lm."""
        lmax = self.lmax if lmax is None else int(lmax)
        P = self.plan(lmax)
        B, nf = maps.shape[0], maps.shape[1]
        self.n_SHTs_forward += B * (1 + (nf == 3))
        scale = np.pi / (3. * self.Nside ** 2)
        out = torch.empty((B, nf, P.nalm), dtype=torch.complex128, device=self.device)
        out[:, 0] = P.adjoint(maps[:, 0].contiguous(), 0, scale)
        if nf == 3:
            out[:, 1:] = P.adjoint(maps[:, 1:].contiguous(), 2, scale)
        return out

    # ------------------------------------------------------------------ SHT wrappers
    @timer_func
    def to_lm(self, input_map, lmax=None):
        """Map -> harmonic space (TQU -> TEB for three fields), i.e. ducc0
        adjoint_synthesis times pi/(3 Nside^2) (polyspec/base.py:131-151)."""
        self.n_SHTs_forward += 1 + (len(input_map) == 3)
        assert len(input_map) in [1, 3], "Wrong input shape supplied!"
        if lmax is None:
            lmax = self.lmax
        m, as_torch = self._in(input_map, torch.float64)
        P = self.plan(lmax)
        scale = np.pi / (3. * self.Nside ** 2)
        if len(m) == 3:
            out = torch.empty((3, P.nalm), dtype=torch.complex128, device=self.device)
            out[0] = P.adjoint(m[0:1], 0, scale)[0]
            out[1:] = P.adjoint(m[1:3].reshape(1, 2, -1), 2, scale)[0]
        else:
            out = P.adjoint(m.reshape(1, -1), 0, scale)
        return self._out(out, as_torch)

    @timer_func
    def to_map(self, input_lm, lmax=None):
        """Harmonic -> map space (TEB -> TQU), ducc0 synthesis (polyspec/base.py:154-176)."""
        self.n_SHTs_reverse += 1 + (len(input_lm) == 3)
        assert len(input_lm) in [1, 3], "Wrong input shape supplied!"
        if lmax is None:
            lmax = self.lmax
        assert len(input_lm[0]) == (lmax + 1) * (lmax + 2) // 2, "Wrong number of alm coefficients!"
        a, as_torch = self._in(input_lm, torch.complex128)
        P = self.plan(lmax)
        if len(a) == 3:
            out = torch.empty((3, self.Npix), dtype=torch.float64, device=self.device)
            out[0] = P.synthesis(a[0:1], 0)[0]
            out[1:] = P.synthesis(a[1:3].reshape(1, 2, -1), 2)[0]
        else:
            out = P.synthesis(a.reshape(1, -1), 0)
        return self._out(out, as_torch)

    @timer_func
    def to_lm_vec(self, input_vec, spin=0, lmax=None):
        """Vector of spin-0 maps, or a [(+s), (-s)] pair of map vectors, to harmonic
        space (polyspec/base.py:179-209)."""
        self.n_SHTs_forward += len(input_vec)
        if lmax is None:
            lmax = self.lmax
        P = self.plan(lmax)
        scale = np.pi / (3. * self.Nside ** 2)
        if spin == 0:
            m, as_torch = self._in(input_vec, torch.float64)
            return self._out(P.adjoint(m, 0, scale), as_torch)
        assert spin > 0, "Spin must be positive!"
        assert len(input_vec) == 2, "Must input both +s and -s maps"
        v, as_torch = self._in(input_vec, torch.complex128)
        map_inputs = _to_real_imag(v[0], v[1])  # [n, 2, npix]
        lm = P.adjoint(map_inputs.contiguous(), int(spin), scale)
        return self._out(_to_plus_minus_complex(lm, spin), as_torch)

    @timer_func
    def to_map_vec(self, input_lm_vec, output_spin=0, lmax=None):
        """Vector of spin-0 alm to maps; for output_spin != 0 the (+s, -s) maps
        of the spin-s transform of [-a, 0] (polyspec/base.py:212-232)."""
        self.n_SHTs_reverse += len(input_lm_vec)
        if lmax is None:
            lmax = self.lmax
        assert len(input_lm_vec[0]) == (lmax + 1) * (lmax + 2) // 2, "Wrong number of alm coefficients!"
        a, as_torch = self._in(input_lm_vec, torch.complex128)
        P = self.plan(lmax)
        if output_spin == 0:
            return self._out(P.synthesis(a, 0), as_torch)
        inp = torch.stack([-a, torch.zeros_like(a)], dim=1)
        out = P.synthesis(inp, int(output_spin))
        return self._out(_to_plus_minus(out), as_torch)

    @timer_func
    def to_lm_spin(self, input_map_plus, input_map_minus, spin, lmax=None):
        """(+s, -s) maps -> (+s, -s) harmonics, HEALPix conventions (polyspec/base.py:235-258)."""
        assert spin > 0, "Spin must be positive!"
        assert type(spin) == int, "Spin must be an integer!"
        self.n_SHTs_forward += 1
        if lmax is None:
            lmax = self.lmax
        p, as_torch = self._in(input_map_plus, torch.complex128)
        mi, _ = self._in(input_map_minus, torch.complex128)
        map_inputs = torch.stack([((p + mi) / 2.).real, ((p - mi) / 2j).real]).reshape(1, 2, -1)
        P = self.plan(lmax)
        lm = P.adjoint(map_inputs.contiguous(), spin, np.pi / (3. * self.Nside ** 2))[0]
        lm_plus = -(lm[0] + 1.0j * lm[1])
        lm_minus = -1 * (-1) ** spin * (lm[0] - 1.0j * lm[1])
        return self._out(torch.stack([lm_plus, lm_minus]), as_torch)

    @timer_func
    def to_map_spin(self, _input_lm_plus, _input_lm_minus, spin, lmax=None):
        """(+s, -s) harmonics -> (+s, -s) maps, HEALPix conventions (polyspec/base.py:261-288)."""
        ap, as_torch = self._in(_input_lm_plus, torch.complex128)
        am, _ = self._in(_input_lm_minus, torch.complex128)
        assert spin > 0, "Spin must be positive!"
        assert type(spin) == int, "Spin must be an integer!"
        self.n_SHTs_reverse += 1
        if lmax is None:
            lmax = self.lmax
        assert len(ap) == (lmax + 1) * (lmax + 2) // 2, "Wrong number of alm coefficients!"
        sgn = (-1) ** spin
        lm_inputs = torch.stack([-(ap + sgn * am) / 2., -(ap - sgn * am) / 2j]).reshape(1, 2, -1)
        P = self.plan(lmax)
        mo = P.synthesis(lm_inputs.contiguous(), spin)[0]
        map_plus = mo[0] + 1.0j * mo[1]
        map_minus = mo[0] - 1.0j * mo[1]
        return self._out(map_plus, as_torch), self._out(map_minus, as_torch)

    def compute_spin_transform_map(self, a_lms, spin, lmax=None):
        """sum_lm sY_lm a_lm for scalar a_lm, spin s = +-1, +-2 (polyspec/base.py:290-297)."""
        if spin > 0:
            return [self.to_map_spin(a_lm, (-1.) ** spin * a_lm, int(abs(spin)), lmax=lmax)[0] for a_lm in a_lms]
        if spin < 0:
            return [self.to_map_spin((-1.) ** spin * a_lm, a_lm, int(abs(spin)), lmax=lmax)[1] for a_lm in a_lms]

    def safe_divide(self, x, y):
        """Divide maps without zero errors."""
        out = np.zeros_like(x)
        out[y != 0] = x[y != 0] / y[y != 0]
        return out

    # ------------------------------------------------------------------ simulations
    def _synalm(self, Cl_input, rng, seed):
        nfield = 1 + 2 * self.pol
        if self.pol:
            rows = [Cl_input['TT'], Cl_input['TE'], Cl_input['TB'], Cl_input['EE'], Cl_input['EB'], Cl_input['BB']]
        else:
            rows = [Cl_input['TT']]
        if rng == 'numpy':
            return torch.as_tensor(synalm_numpy(rows, self.lmax, nfield), device=self.device)
        # device generator (Philox): same distribution, different stream
        g = torch.Generator(device=self.device)
        g.manual_seed(int(seed) if seed is not None else int(torch.randint(0, 2 ** 62, (1,))))
        key = ('sqrtC', id(Cl_input), self.lmax)
        S = self._dev_cache.get(key)
        if S is None:
            C = np.zeros((self.lmax + 1, nfield, nfield))
            k = 0
            for i in range(nfield):
                for j in range(i, nfield):
                    C[:, i, j] = C[:, j, i] = np.asarray(rows[k])[:self.lmax + 1]
                    k += 1
            w, V = np.linalg.eigh(C)
            Sn = np.einsum("lij,lj,lkj->lik", V, np.sqrt(np.clip(w, 0.0, None)), V)
            S = torch.as_tensor(Sn, device=self.device)
            self._dev_cache[key] = S
        n = len(self.l_arr)
        z = torch.randn((nfield, n, 2), dtype=torch.float64, device=self.device, generator=g)
        mpos = self.dev('m_weight') > 1
        zc = torch.where(mpos[None], torch.complex(z[..., 0], z[..., 1]) / np.sqrt(2.0),
                         torch.complex(z[..., 0], torch.zeros_like(z[..., 0])))
        Sl = S[self.dev('l_arr')]  # [n, f, f]
        return torch.einsum("nij,jn->in", Sl.to(torch.complex128), zc)

    def generate_data(self, seed=None, Cl_input={}, output_type='map', deconvolve_beam=False, b_input=None,
                      add_B=False, remove_mean=True, sum_ells='even', lmax=None, rng='numpy'):
        """Gaussian (optionally bispectrum-weighted) simulation (polyspec/base.py:305-422).

        ``rng='numpy'`` draws from numpy's global generator after
        ``np.random.seed(seed)``, as the reference does; ``rng='device'`` draws
        on the GPU (Philox) from ``seed``.  Returns numpy arrays for
        ``rng='numpy'`` and CUDA tensors for ``rng='device'``.
        """
        assert output_type in ['harmonic', 'map'], "Valid output types are 'harmonic' and 'map' only!"
        as_torch = rng == 'device'
        if seed is not None and rng == 'numpy':
            np.random.seed(seed)
        if lmax is None:
            lmax = self.lmax
        if len(Cl_input.keys()) == 0:
            Cl_input = self.Cl_tot
        if self.pol:
            assert len(Cl_input.keys()) == 6 or len(Cl_input.keys()) == 4, \
                "Need to specify {ClTT, ClEE, ClBB, ClTE} and optionally {ClTB, ClEB}."
            if len(Cl_input.keys()) == 4:
                Cl_input['TB'] = Cl_input['EB'] = 0. * Cl_input['TT']
        initial_lm = self._synalm(Cl_input, rng, seed)
        lfilt = torch.as_tensor(self.l_arr <= lmax, device=self.device)
        initial_lm = initial_lm[:, lfilt]
        if not add_B:
            if deconvolve_beam:
                this_beam = self.dev('beam_lm', lmax)
                initial_lm = torch.where(this_beam != 0, initial_lm / torch.where(this_beam != 0, this_beam, 1.0),
                                         torch.zeros_like(initial_lm))
            if output_type == 'map':
                return self._out(self.to_map(initial_lm, lmax=lmax), as_torch)
            return self._out(initial_lm, as_torch)

        # bispectrum-weighted field (Smith & Zaldarriaga 2006), polyspec/base.py:345-422
        Cinv_lm = torch.einsum('ijk,jk->ik', self.dev('inv_Cl_tot_lm_mat'), initial_lm)
        bl = torch.as_tensor(np.asarray(b_input(self.l_arr)), device=self.device)
        bCinv_lm = sum(bl[i] * Cinv_lm[i] for i in range(len(Cinv_lm)))
        sgn = torch.tensor([[1.], [-1.]], dtype=torch.float64, device=self.device)
        bCinv_map_pm1 = torch.stack(self.to_map_spin(bCinv_lm, -bCinv_lm, 1)) * sgn
        bCinv_map_pm2 = torch.stack(self.to_map_spin(bCinv_lm, bCinv_lm, 2))
        tmp_lm = self.to_lm_spin(bCinv_map_pm1[0] * bCinv_map_pm1[0], bCinv_map_pm1[1] * bCinv_map_pm1[1], 2).flip(0)
        tmp_lm = tmp_lm - 2 * sgn * self.to_lm_spin(bCinv_map_pm1[1] * bCinv_map_pm2[0],
                                                    -bCinv_map_pm1[0] * bCinv_map_pm2[1], 1)
        if sum_ells == 'even':
            tmp_lm = (tmp_lm[0] + tmp_lm[1]) / 2.
        elif sum_ells == 'odd':
            tmp_lm = 1.0j * (tmp_lm[0] - tmp_lm[1]) / 2.
        elif sum_ells == 'both':
            tmp_lm = (1. + 1.0j) * tmp_lm[0] / 2. + (1 - 1.0j) / 2. * tmp_lm[1]
        else:
            raise Exception("Unknown value of sum_ells supplied")
        grad_lm = [1. / 6. * tmp_lm * bl[i] for i in range(len(Cinv_lm))]
        output_lm = torch.stack([initial_lm[i] + 1. / 3. * grad_lm[i] for i in range(len(Cinv_lm))])
        if deconvolve_beam:
            this_beam = self.dev('beam_lm', lmax)
            output_lm = torch.where(this_beam != 0, output_lm / torch.where(this_beam != 0, this_beam, 1.0),
                                    torch.zeros_like(output_lm))
        output_map = self.to_map(output_lm)
        if remove_mean:
            if not hasattr(self, 'map_offset') or (hasattr(self, 'map_offset') and self.saved_spec != [Cl_input, b_input]):
                print("Computing offset for synthetic maps")
                map_offset = 0.
                for ii in range(100):
                    map_offset += self.generate_data(Cl_input=Cl_input, b_input=b_input, seed=int(1e6) + ii, add_B=True,
                                                     remove_mean=False, deconvolve_beam=deconvolve_beam,
                                                     rng='device') / 100.
                self.map_offset = map_offset
                self.saved_spec = [Cl_input, b_input]
            output_map = output_map - self.map_offset
        if output_type == 'harmonic':
            return self._out(self.to_lm(output_map), as_torch)
        return self._out(output_map, as_torch)

    def applyAinv(self, input_map, input_type='map', lmax=-1):
        """Exact inverse weighting B C_tot^-1 B of beam-deconvolved GRFs (polyspec/base.py:424-446)."""
        if lmax == -1:
            lmax = self.lmax
        assert input_type in ['harmonic', 'map'], "Valid input types are 'harmonic' and 'map' only!"
        if input_type == 'map':
            x, as_torch = self._in(input_map, torch.float64)
            input_map_lm = self.to_lm(x, lmax=lmax)
        else:
            input_map_lm, as_torch = self._in(input_map, torch.complex128)
        b = self.dev('beam_lm', lmax)
        out = b * torch.einsum('ijk,jk->ik', self.dev('inv_Cl_tot_lm_mat', lmax), b * input_map_lm)
        return self._out(out, as_torch)


# ---------------------------------------------------------------------- recombinations
# numpy / torch forms of ideal_fisher.pyx to_plus_minus, to_plus_minus_complex,
# to_real_imag (polyspec/cython/ideal_fisher.pyx:237-320)
def _to_plus_minus(map):
    """map[n, 2, npix] (Re, Im) -> [2, n, npix]: (Re + i Im, Re - i Im)."""
    return torch.stack([map[:, 0] + 1.0j * map[:, 1], map[:, 0] - 1.0j * map[:, 1]])


def _to_plus_minus_complex(map, spin):
    """alm[n, 2, nlm] (G, C) -> [2, n, nlm]: (-(G + iC), -(-1)^s (G - iC))."""
    return torch.stack([-(map[:, 0] + 1.0j * map[:, 1]), -(-1.) ** spin * (map[:, 0] - 1.0j * map[:, 1])])


def _to_real_imag(mapP, mapM):
    """(+, -) maps [n, npix] -> [n, 2, npix]: (Re (P + M)/2, Im (P - M)/2)."""
    return torch.stack([((mapP + mapM) / 2.).real, ((mapP - mapM) / 2.).imag], dim=1)
