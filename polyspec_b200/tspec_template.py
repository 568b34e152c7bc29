"""Template trispectrum estimator on the GPU (mirror of polyspec/tspec_template.py)
for the gNL-loc, gNL-con, EFTI (gNL-dotdot, gNL-dotdel, gNL-deldel), tauNL-loc,
direction-dependent tauNL-direc:n1,n3,n, tauNL-even:n, tauNL-odd:n, collider
tauNL-light:s,nu_s and tauNL-heavy:s,mu_s, lensing and point-source templates.

``TSpecTemplate(base, mask, applySinv, templates, k_arr, Tl_arr, lmin, lmax, ...)``
keeps the reference constructor, its checks and attributes (l- and L-ranges and
filters, ``to_compute``, ``p_inds``, ``qlXs``, ``plLXs``, ``rlXs``, ``alXs``,
``blXs``, ``clXs``, ``timers``), the
simulation handling (``generate_sims``, ``load_sims``) and the estimator methods
(``Tl_numerator``, ``compute_fisher_contribution``, ``compute_fisher``,
``Tl_unwindowed``, ``report_timings``, ``reset_timings``).  The radial-sampling
optimisers raise NotImplementedError.

``applySinv`` receives and returns CUDA tensors (as for PSpecBin/BSpecBin here);
one with a ``.batched`` method filters the 4 x n_templates Q rows of the Fisher
contribution in one batch.  Returned numerators and Fisher matrices are numpy.

Device mapping:
* k-space integrals (polyspec/tspec_template.py:520-708): the j_l(x) table on the
  reference's x grid and the q, p, r (radial) and a, b, c ((r, tau)) trapezium
  sums run as the ``ps_kint_*`` kernels (same grid, interpolation and summation
  order; b with j_l' from the interpolated j_{l-1}, j_{l+1}).
* Filtered maps: ``ps_apply_fl_weights`` then one batched spin-0 synthesis over
  the radial samples (P, Q, R, A, B maps; C is spin 1); the lensing U and V maps
  are spin 0/1/2/3 syntheses; Phi_LM is the lens_phi_sum kernel plus one spin-1
  adjoint.
* tauNL-loc: F_L(r, r') from ``ps_tau_F_integral`` (closed form, as the reference);
  the (P Q)_LM maps are a product kernel plus a batched adjoint to Lmax; the sum
  over (L, M, r, r') and the F-convolution of the Fisher derivative are
  ``ps_tau_convolve_F``.
* Collider templates: the complex p^beta integrals are ``ps_kint_radial`` on the real
  and imaginary parts of the k-weight, F^beta is ``ps_kint_collider_jlK`` +
  ``ps_kint_collider_F``; the tau sums are ``ps_tau_sum_collider_diag`` (s = 0 and
  nu_s = 0) and ``ps_tau_sum_collider_general``; the Fisher derivative convolves with
  ``ps_convolve_F_collider`` and shifts with ``ps_pF_map_complex``.
* Numerators: the radial pixel sums ``gnl_*(_disc)_sum``; lensing and point
  source sums are device reductions.
* Fisher: the ``multiply*`` products, a batched spin-0 or spin-1 adjoint over the
  samples and ``ps_radial_sum_lm`` for the gNL Q derivatives; spin-1/2/3 adjoints
  for lensing; the batched S^-1 weighting; the Fisher outer product.
"""
import ctypes
import time

import numpy as np
import torch

from . import _lib, pixel

SUPPORTED = ['gNL-loc', 'gNL-con', 'gNL-dotdot', 'gNL-dotdel', 'gNL-deldel', 'tauNL-loc', 'lensing',
             'point-source']


def _is_direc(t):
    """Direction-dependent tauNL templates: tauNL-direc:n1,n3,n, tauNL-even:n and tauNL-odd:n."""
    return any(s in t for s in ('tauNL-direc', 'tauNL-even', 'tauNL-odd'))


def _is_coll(t):
    """Collider templates: tauNL-light:s,nu_s and tauNL-heavy:s,mu_s."""
    return 'tauNL-light' in t or 'tauNL-heavy' in t


def _coll_parse(t):
    a, b = t.split(':')[1].split(',')
    return int(a), float(b)


def _ckey(beta):
    """Key of the collider P^beta maps of one filtered field (polyspec/tspec_template.py:1089)."""
    return 'coll-%.8f,%.8fi' % (np.real(beta), np.imag(beta))


def _ckey_s(s, beta):
    """Key of the collider [P^beta_{s,lam} Q] harmonic maps (polyspec/tspec_template.py:1246)."""
    return 'coll-%d,%.8f,%.8fi' % (s, np.real(beta), np.imag(beta))


def _fact_ratio(num, den):
    """prod(num)! / prod(den)! as a float, from exact integers."""
    from math import factorial
    a, b = 1, 1
    for x in num:
        a *= factorial(x)
    for x in den:
        b *= factorial(x)
    return a / b


def wig3zero(l1, l2, l3):
    """Wigner 3j symbol (l1 l2 l3; 0 0 0) for small integer l (the closed form of Edmonds 1957, eq. 3.7.17)."""
    L = l1 + l2 + l3
    if L % 2 or l3 < abs(l1 - l2) or l3 > l1 + l2 or min(l1, l2, l3) < 0:
        return 0.
    g = L // 2
    r = np.sqrt(_fact_ratio((L - 2 * l1, L - 2 * l2, L - 2 * l3), (L + 1,)))
    return (-1.) ** g * r * _fact_ratio((g,), (g - l1, g - l2, g - l3))


def wig3(j1, j2, j3, m1, m2, m3):
    """Wigner 3j symbol (j1 j2 j3; m1 m2 m3) for small integer j (Racah's single sum, Edmonds 1957, eq. 3.7.3)."""
    if m1 + m2 + m3 != 0 or j3 < abs(j1 - j2) or j3 > j1 + j2 or abs(m1) > j1 or abs(m2) > j2 or abs(m3) > j3:
        return 0.
    delta = np.sqrt(_fact_ratio((j1 + j2 - j3, j1 - j2 + j3, -j1 + j2 + j3, j1 + m1, j1 - m1, j2 + m2, j2 - m2,
                                 j3 + m3, j3 - m3), (j1 + j2 + j3 + 1,)))
    from fractions import Fraction
    from math import factorial
    total = Fraction(0)  # exact, so that symbols that vanish by cancellation are 0
    for k in range(max(0, j2 - j3 - m1, j1 - j3 + m2), min(j1 + j2 - j3, j1 - m1, j2 + m2) + 1):
        den = 1
        for x in (k, j1 + j2 - j3 - k, j1 - m1 - k, j2 + m2 - k, j3 - j2 + m1 + k, j3 - j1 - m2 + k):
            den *= factorial(x)
        total += Fraction((-1) ** k, den)
    return (-1.) ** (j1 - j2 - m3) * delta * float(total)


def wig6(j1, j2, j3, j4, j5, j6):
    """Wigner 6j symbol {j1 j2 j3; j4 j5 j6} for small integer j (Racah's single sum, Edmonds 1957, eq. 6.3.7)."""
    triads = ((j1, j2, j3), (j1, j5, j6), (j4, j2, j6), (j4, j5, j3))
    for a, b, c in triads:
        if c < abs(a - b) or c > a + b or min(a, b, c) < 0:
            return 0.
    delta = 1.
    for a, b, c in triads:
        delta *= np.sqrt(_fact_ratio((a + b - c, a - b + c, -a + b + c), (a + b + c + 1,)))
    A = [a + b + c for a, b, c in triads]
    B = (j1 + j2 + j4 + j5, j2 + j3 + j5 + j6, j3 + j1 + j6 + j4)
    total = 0.
    for t in range(max(A), min(B) + 1):
        total += (-1.) ** t * _fact_ratio((t + 1,), [t - a for a in A] + [b - t for b in B])
    return delta * total


def _vp(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


class TSpecTemplate:
    def __init__(self, base, mask, applySinv, templates, k_arr, Tl_arr, lmin, lmax,
                 Lmin=None, Lmax=None, Lmin_lens=None, Lmax_lens=None, ns=0.96, As=2.1e-9, k_pivot=0.05,
                 r_values=[], r_weights={}, rtau_values=[], rtau_weights={},
                 C_phi=[], C_lens_weight={}, K_coll=0.1, k_coll=0.1, r_star=None, r_hor=None):
        self.base = base
        self.mask = mask
        self.applySinv = applySinv
        self.pol = self.base.pol
        self.templates = templates
        self.k_arr = k_arr
        self.lmin = lmin
        self.lmax = lmax
        self.ns = ns
        self.As = As
        self.k_pivot = k_pivot
        self.K_coll = K_coll
        self.k_coll = k_coll

        print("Primordial Spectrum: n_s = %.3f, A_s = %.3e, k_pivot = %.3f" % (self.ns, self.As, self.k_pivot))
        self.Pzeta = lambda k: 2. * np.pi ** 2. / k ** 3 * self.As * (k / self.k_pivot) ** (self.ns - 1)

        assert self.lmax <= base.lmax, "Maximum l can't be larger than HEALPix resolution!"
        assert self.lmin >= 2, "Minimum l can't be less than 2"
        if self.lmax > (base.lmax + 1) * 2 / 3:
            print("## Caution: Maximum l is greater than (2/3)*HEALPix-lmax; this might cause boundary effects.")
        self.Lmin = 1 if Lmin is None else Lmin
        self.Lmax = min([base.lmax, 2 * self.lmax]) if Lmax is None else Lmax
        assert self.Lmin >= 1, "Minimum L can't be less than 1"
        assert self.Lmax <= 2 * self.lmax, "Lmax <= 2*lmax by the triangle conditions"
        assert self.Lmax <= base.lmax, "Maximum L can't be larger than HEALPix resolution"

        # lensing L ranges (polyspec/tspec_template.py:95-116)
        if 'lensing' in self.templates:
            gnl = np.any(['gNL' in t for t in self.templates])
            tau = np.any(['tauNL' in t for t in self.templates])
            if Lmin_lens is None:
                self.Lmin_lens = 1 if (gnl or not tau) else self.Lmin
            else:
                self.Lmin_lens = Lmin_lens
            if Lmax_lens is None:
                self.Lmax_lens = min([base.lmax, 2 * self.lmax]) if (gnl or not tau) else self.Lmax
            else:
                self.Lmax_lens = Lmax_lens
            assert self.Lmin_lens >= 1, "Minimum L_lens can't be less than 1"
            assert self.Lmax_lens <= 2 * self.lmax, "Lmax_lens <= 2*lmax by the triangle conditions"
            assert self.Lmax_lens <= base.lmax, "Maximum L can't be larger than HEALPix resolution"

        self.lfilt = (self.base.l_arr >= self.lmin) & (self.base.l_arr <= self.lmax)
        self.Lfilt = (self.base.l_arr >= self.Lmin) & (self.base.l_arr <= self.Lmax)
        self.ls, self.ms = self.base.l_arr[self.lfilt], self.base.m_arr[self.lfilt]
        if 'lensing' in self.templates:
            self.Lfilt_lens = (self.base.l_arr >= self.Lmin_lens) & (self.base.l_arr <= self.Lmax_lens)
        self.m_weight = np.asarray(self.base.m_weight[self.lfilt], order='C')
        self.Cinv = np.asarray(self.base.inv_Cl_tot_lm_mat[:, :, self.lfilt], order='C')
        self.beam_lm = np.asarray(self.base.beam_lm)[:, self.lfilt]

        print("l-range: %s" % [self.lmin, self.lmax])
        if 'lensing' in self.templates:
            print("Lensing L-range: %s" % [self.Lmin_lens, self.Lmax_lens])
        print("Polarizations: ['T', 'E']" if self.pol else "Polarizations: ['T']")

        self._configure_templates(templates, C_phi, C_lens_weight)

        if not type(mask) == float or type(mask) == int:
            if len(mask) == 1 or len(mask) == 3:
                assert len(mask[0]) == self.base.Npix, f'Mask has incorrect shape: {np.shape(mask)}'
            else:
                assert len(mask) == self.base.Npix, f'Mask has incorrect shape: {np.shape(mask)}'
        if np.std(self.mask) < 1e-12 and np.abs(np.mean(self.mask) - 1) < 1e-12:
            print("Mask: ones")
            self.ones_mask = True
        else:
            print("Mask: spatially varying")
            self.ones_mask = False

        self.r_star = 13882.607764400758 if r_star is None else r_star
        self.r_hor = 14163.032903769747 if r_hor is None else r_hor

        if self.ints_1d or self.ints_2d:
            self.Tl_arr = np.asarray(Tl_arr, dtype=np.float64, order='C')
            if not self.pol:
                assert len(self.Tl_arr) == 1, "Transfer function should contain only T components"
            else:
                assert len(self.Tl_arr) == 2, "Transfer function should contain both T and E components"
            assert len(self.Tl_arr[0]) >= self.lmax + 1, "Transfer function must contain all ell modes of interest"
            assert self.Tl_arr[0][:2].sum() == 0., "Transfer function should return zero for ell = 0, 1"
            assert len(self.Tl_arr[0][0]) == len(k_arr), "Transfer function must be computed on the input k-grid"
            if self.pol:
                assert self.Tl_arr[1][:2].sum() == 0., "Transfer function should return zero for ell = 0, 1"

        self.timers = {x: 0. for x in ['precomputation', 'numerator', 'fisher', 'optimization', 'analytic_fisher',
                                       'fish_grfs', 'fish_outer', 'fish_weighting', 'fish_convolve', 'fish_deriv',
                                       'fish_products', 'Sinv', 'Ainv', 'map_transforms', 'gNL_summation',
                                       'tauNL_products', 'tauNL_summation', 'lensing_products',
                                       'lensing_summation']}
        self.base.time_sht = 0.

        if len(r_values) == 0 and self.ints_1d:
            print("# No input radial sampling points supplied; these can be computed with the "
                  "optimize_radial_sampling_1d() function\n")
            self.N_r = 0
        elif self.ints_1d:
            print("Reading in precomputed radial integration points")
            assert len(r_values) > 0, "Must supply radial sampling points!"
            for t in templates:
                if t in self.all_templates_1d or _is_direc(t):
                    assert t in r_weights.keys(), "Must supply weight for template %s" % t
            self.r_arr = np.asarray(r_values, dtype=np.float64)
            self.N_r = len(self.r_arr)
            self.r_weights = r_weights
        else:
            self.N_r = 0
        if len(rtau_values) == 0 and self.ints_2d:
            print("# No input r/tau sampling points supplied; these can be computed with the "
                  "optimize_radial_sampling_2d() function\n")
            self.N_rtau = 0
        elif self.ints_2d:
            print("Reading in precomputed r/tau integration points")
            assert len(rtau_values) > 0 and len(rtau_values[0]) == 2, \
                "Must supply r/tau sampling points for 2d integrals shapes!"
            for t in templates:
                if t in self.all_templates_2d:
                    assert t in rtau_weights.keys(), "Must supply weight for template %s" % t
            self.rtau_arr = np.asarray(rtau_values, dtype=np.float64)
            self.N_rtau = len(self.rtau_arr)
            assert max(self.rtau_arr[:, 0]) >= 0, "r should be in range (0, inf)"
            assert max(self.rtau_arr[:, 1]) <= 0, "tau should be in range (-inf, 0)"
            self.rtau_weights = rtau_weights
        else:
            self.N_rtau = 0

        dev = base.device
        self._dev = dev
        self.d_lfilt = torch.as_tensor(np.nonzero(self.lfilt)[0], device=dev)
        self.d_lminfilt = torch.as_tensor(np.nonzero(self.lminfilt)[0], device=dev)
        self.d_beam_lm = torch.as_tensor(np.ascontiguousarray(self.beam_lm), device=dev)
        self.d_m_weight = torch.as_tensor(self.m_weight, device=dev)
        self.d_mask = torch.as_tensor(np.asarray(mask, dtype=np.float64), device=dev)
        if self.d_mask.dim() == 1:
            self.d_mask = self.d_mask[None]
        if 'lensing' in self.templates:
            self.d_Lminfilt_lens = torch.as_tensor(np.nonzero(self.Lminfilt_lens)[0], device=dev)
        t0 = time.time()
        if self.N_r > 0:
            self._prepare_templates(self.ints_1d, False, self.ints_coll)
        if self.N_rtau > 0:
            self._prepare_templates(False, self.ints_2d, False)
        self.timers['precomputation'] += time.time() - t0

    # ------------------------------------------------------------------ configuration
    def _configure_templates(self, templates, C_phi, C_lens_weight):
        """Template bookkeeping (polyspec/tspec_template.py:243-451) for the supported templates."""
        self.all_templates_1d = ['gNL-loc', 'gNL-con', 'tauNL-loc', 'tauNL-direc', 'tauNL-even', 'tauNL-odd']
        self.all_templates_2d = ['gNL-dotdot', 'gNL-dotdel', 'gNL-deldel']
        self.all_templates_coll = ['tauNL-light', 'tauNL-heavy']
        self.all_templates = self.all_templates_1d + self.all_templates_2d + self.all_templates_coll + \
            ['lensing', 'point-source']
        for t in templates:
            known = t in self.all_templates or any(s in t for s in ('tauNL-direc', 'tauNL-even', 'tauNL-odd',
                                                                     'tauNL-light', 'tauNL-heavy'))
            assert known, "Unknown template %s supplied!" % t
            if t not in SUPPORTED and not _is_direc(t) and not _is_coll(t):
                raise NotImplementedError("template %s is not implemented by the CUDA backend (supported: %s, "
                                          "tauNL-direc:n1,n3,n, tauNL-even:n, tauNL-odd:n, tauNL-light:s,nu_s, "
                                          "tauNL-heavy:s,mu_s)" % (t, SUPPORTED))
        print("Templates: %s" % templates)
        self.ints_1d, self.ints_2d, self.ints_coll = False, False, False
        self.to_compute, self.n1n3n, self.coll_params = [], [], {}
        if any(_is_coll(t) for t in templates):
            assert self.K_coll <= self.k_coll, "Collider K_cut can't exceed collider k_cut"
            print("Collider k-range: K < %.2e, k > %.2e" % (self.K_coll, self.k_coll))
        if 'gNL-loc' in templates:
            self.to_compute.append(['q'])
            self.ints_1d = True
        if 'gNL-con' in templates:
            self.to_compute.append(['r'])
            self.ints_1d = True
        if 'gNL-dotdot' in templates:
            self.to_compute.append(['a'])
            self.ints_2d = True
        if 'gNL-dotdel' in templates:
            self.to_compute.append(['a', 'b', 'c'])
            self.ints_2d = True
        if 'gNL-deldel' in templates:
            self.to_compute.append(['b', 'c'])
            self.ints_2d = True
        n1n3n = []
        if 'tauNL-loc' in templates:
            self.to_compute.append(['q'])
            n1n3n.append([0, 0, 0])
            self.ints_1d = True
        for t in templates:
            if 'tauNL-direc' in t:
                n1, n3, n = np.asarray(t.split(':')[1].split(','), dtype=int)
                if n1 == 0 and n3 == 0 and n == 0 and 'tauNL-loc' in self.templates:
                    raise Exception("tauNL-loc and tauNL-direc:0,0,0 are fully degenerate!")
                if ('tauNL-direc:%d,%d,%d' % (n3, n1, n) in self.templates) and (n1 < n3):
                    raise Exception("tauNL-direc:%d,%d,%d and tauNL-direc:%d,%d,%d are fully degenerate!"
                                    % (n1, n3, n, n3, n1, n))
                assert (n >= abs(n1 - n3)) and (n <= n1 + n3), \
                    "Direction-dependent indices %d,%d,%d do not satisfy triangle conditions" % (n1, n3, n)
                assert (n1 <= 5) and (n3 <= 5) and (n <= 5), "n>5 has not yet been implemented!"
                self.to_compute.append(['q'])
                n1n3n.append([int(n1), int(n3), int(n)])
                self.ints_1d = True
            if 'tauNL-even' in t:
                n = int(t.split(':')[1])
                if n == 0 and 'tauNL-loc' in self.templates:
                    raise Exception("tauNL-even:0 and tauNL-loc are fully degenerate!")
                if n == 0 and 'tauNL-direc:0,0,0' in self.templates:
                    raise Exception("tauNL-even:0 and tauNL-direc:0,0,0 are fully degenerate!")
                if ('tauNL-direc:%d,%d,%d' % (0, n, n) in self.templates) and \
                        ('tauNL-direc:%d,%d,%d' % (n, n, 0) in self.templates):
                    raise Exception("tauNL-even:%d is fully degenerate with tauNL-direc:%d,%d,%d and "
                                    "tauNL-direc:%d,%d,%d" % (n, 0, n, n, n, n, 0))
                self.to_compute.append(['q'])
                n1n3n += [[0, n, n], [n, n, 0]]
                self.ints_1d = True
            if 'tauNL-odd' in t:
                n = int(t.split(':')[1])
                if n == 0 and 'tauNL-direc:1,1,1' in self.templates:
                    raise Exception("tauNL-odd:0 and tauNL-direc:1,1,1 are fully degenerate!")
                # (n1, n3, n) pieces that satisfy the triangle conditions (polyspec/tspec_template.py:329-345)
                cands = [[n - 1, n - 1, 1], [n - 1, n + 1, 1], [n + 1, n - 1, 1], [n + 1, n + 1, 1],
                         [n - 1, 1, n - 1], [n - 1, 1, n + 1], [n + 1, 1, n - 1], [n + 1, 1, n + 1],
                         [1, n - 1, n - 1], [1, n - 1, n + 1], [1, n + 1, n - 1], [1, n + 1, n + 1]]
                n1n3n += [c for c in cands if abs(c[0] - c[1]) <= c[2] <= c[0] + c[1] and min(c) >= 0]
                self.to_compute.append(['q'])
                self.ints_1d = True
            if 'tauNL-light' in t:
                # light particle of spin s and nu_s (polyspec/tspec_template.py:347-371): beta = nu_s - 3/2
                s, nu_s = _coll_parse(t)
                if s == 0 and nu_s == 1.5 and ('tauNL-loc' in self.templates):
                    raise Exception("tauNL-loc and tauNL-light:0,1.5 are fully degenerate!")
                if nu_s == 1.5 and ('tauNL-direc:%d,%d,0' % (s, s) in self.templates):
                    raise Exception("tauNL-direc:%d,%d,0 and tauNL-light:%d,1.5 are fully degenerate!" % (s, s, s))
                if s == 0:
                    assert 0. <= nu_s <= 1.5, "Light spin-0 particles have nu_s in (0, 3/2)"
                else:
                    assert 0 <= nu_s <= s - 0.5, "Light spin-%d particles have nu_s in (0, %.1f)" % (s, s - 1. / 2.)
                    if nu_s > 0.5:
                        print("## Warning: Spin = %d nu_s = %d violates the Higuchi bound!" % (s, nu_s))
                self._merge_coll({nu_s - 3. / 2.: [[s, S] for S in range(0, 2 * s + 1, 2)]})
                self.to_compute.append(['q'])
                self.ints_coll = True
                self.ints_1d = True
            if 'tauNL-heavy' in t:
                # heavy particle of spin s and mass mu_s (:372-389): beta = -3/2 +- i mu_s
                s, mu_s = _coll_parse(t)
                if mu_s == 0 and ('tauNL-light:%d,%s' % (s, mu_s) in self.templates):
                    raise Exception("tauNL-light:s,0 and tauNL-heavy:s,0 are fully degenerate!")
                assert mu_s >= 0., "Heavy spin-0 particles have mu_s >=0"
                params = [[s, S] for S in range(0, 2 * s + 1, 2)]
                self._merge_coll({1.0j * mu_s - 3. / 2.: params, -1.0j * mu_s - 3. / 2.: params})
                self.to_compute.append(['q'])
                self.ints_coll = True
                self.ints_1d = True
        for t in templates:
            if 'lensing' in t:
                assert len(C_phi) > 0, "Must supply lensing power spectrum!"
                assert len(C_phi) >= self.Lmax_lens + 1, "Must specify C^phi-phi(L) up to at least Lmax."
                if not self.pol:
                    assert 'TT' in C_lens_weight.keys(), "Must specify unlensed TT power spectrum!"
                else:
                    assert 'TE' in C_lens_weight.keys(), "Must specify unlensed TE power spectrum!"
                    assert 'EE' in C_lens_weight.keys(), "Must specify unlensed EE power spectrum!"
                    assert 'BB' in C_lens_weight.keys(), "Must specify unlensed BB power spectrum!"
                    for k in C_lens_weight.keys():
                        assert len(C_lens_weight[k]) >= self.lmax + 1, \
                            "Must specify C_lens_weight(l) up to at least lmax."
                self.C_phi = C_phi
                self.C_lens_weight = {k: C_lens_weight[k][:self.lmax + 1] for k in C_lens_weight.keys()}
                self.to_compute.append(['u', 'v'])
            if 'point-source' in t:
                self.to_compute.append(['u'])
        self.n1n3n = np.asarray(n1n3n, dtype=int).reshape(-1, 3)
        self.to_compute = np.unique(np.concatenate(self.to_compute)) if self.to_compute else np.array([])
        self.nmax = int(np.max(self.n1n3n[:, :2])) if len(self.n1n3n) > 0 else 0
        self.coll_params = {k: np.asarray(v, dtype=int).reshape(-1, 2) for k, v in self.coll_params.items()}
        self.nmax_coll = int(max([np.max(v[:, 0]) for v in self.coll_params.values()], default=0))
        self.nmax_coll_F = int(max([np.max(v[:, 1]) for v in self.coll_params.values()], default=0))
        self.p_inds = [0] if 'gNL-loc' in self.templates else []
        if len(self.n1n3n) > 0:
            self.p_inds = [int(x) for x in np.unique(self.p_inds + list(np.unique(self.n1n3n[:, :2])))]
        self.nmax_F = int(np.max(self.n1n3n[:, 2])) if len(self.n1n3n) > 0 else 0
        self.nLmax = self.Lmax + max(self.nmax_F, self.nmax_coll_F)
        self.nLmin = self.Lmin - max(self.nmax_F, self.nmax_coll_F)
        # The reference fails later when this does not hold: its default Lmax = min(base.lmax, 2 lmax)
        # (polyspec/tspec_template.py:87-88) plus n > 0 asks to_lm_vec for L beyond base.lmax
        # (:1302), whose output then no longer matches the l <= base.lmax filters (:443-447).
        # Here the configuration is refused at construction, also under python -O.
        if self.nLmax > int(np.max(self.base.l_arr)):
            raise ValueError("Lmax + max(n) = %d exceeds the maps' lmax %d: pass Lmax <= %d"
                             % (self.nLmax, int(np.max(self.base.l_arr)),
                                int(np.max(self.base.l_arr)) - max(self.nmax_F, self.nmax_coll_F)))
        self.nLfilt = (self.base.l_arr >= self.nLmin) & (self.base.l_arr <= self.nLmax)
        self.Ls, self.Ms = self.base.l_arr[self.nLfilt], self.base.m_arr[self.nLfilt]
        self.nLminfilt = self.base.l_arr[self.base.l_arr <= self.nLmax] >= self.nLmin
        self.Lminfilt = self.base.l_arr[self.base.l_arr <= self.Lmax] >= self.Lmin
        if 'lensing' in self.templates:
            self.Lminfilt_lens = self.base.l_arr[self.base.l_arr <= self.Lmax_lens] >= self.Lmin_lens
        self.lminfilt = self.base.l_arr[self.base.l_arr <= self.lmax] >= self.lmin

    def _merge_coll(self, d2):
        """Merge collider (beta -> [[s, S], ..]) entries, dropping duplicates (polyspec/tspec_template.py:262-272)."""
        for key, items in d2.items():
            if key in self.coll_params:
                new = []
                for item in list(items) + list(self.coll_params[key]):
                    if item not in new:
                        new.append(item)
                self.coll_params[key] = new
            else:
                self.coll_params[key] = list(items)

    def _prepare_templates(self, ints_1d=True, ints_2d=False, ints_coll=False):
        """k-space integrals on the GPU (polyspec/tspec_template.py:520-708): p and q (gNL-loc),
        r (gNL-con) on the radial samples; a, b, c (the EFTI shapes) on the (r, tau) samples.
        The j_l(x) table, its x grid, the interpolation to k r and the trapezium rule follow
        the reference; ``ps_kint_bessel_table`` and ``ps_kint_radial`` do the work."""
        dev = self._dev
        print("N_k: %d" % len(self.k_arr))
        if ints_1d:
            print("N_r: %d" % self.N_r)
        if ints_2d:
            print("N_rtau: %d" % self.N_rtau)
        nmax_p = max(self.nmax, self.nmax_coll)
        lmax = max([self.lmax + 1, self.lmax + nmax_p])
        lmin = max([min([self.lmin - 1, self.lmin - nmax_p]), 0])
        print("\nPrecomputing Bessel functions")
        k_arr = np.asarray(self.k_arr, dtype=np.float64)
        max_kr = 0.
        if ints_1d:
            max_kr = max(k_arr) * max([max_kr, max(self.r_arr)])
        if ints_2d:
            max_kr = max(k_arr) * max([max_kr, self.r_hor + 10000 + 5e6])
        x_arr = list(np.arange(0, lmax * 2, 0.01)) + list(np.arange(lmax * 2, min(max_kr * 1.01, lmax * 100), 0.1))
        if max_kr > 100 * lmax:
            x_arr += list(np.linspace(lmax * 100, max_kr * 1.01, 1000))
        x_arr = np.asarray(x_arr, dtype=np.float64)
        d_x = torch.as_tensor(x_arr, device=dev)
        nl_tab = lmax - lmin + 1
        table = torch.empty((nl_tab, len(x_arr)), dtype=torch.float64, device=dev)
        _lib.call("ps_kint_bessel_table", _vp(d_x), len(x_arr), lmin, lmax, _vp(table), _stream())
        if not bool(torch.isfinite(table).all()):
            raise Exception("Spherical Bessel calculation failed!")
        print("Interpolating Bessel functions")
        npol = len(self.Tl_arr)
        npol_out = 1 + 2 * self.pol
        d_k = torch.as_tensor(k_arr, device=dev)
        d_T = torch.as_tensor(np.ascontiguousarray(self.Tl_arr), device=dev)
        nl_T = self.Tl_arr.shape[1]
        Pz = self.Pzeta(k_arr)

        def integral(kprod, r_arr, out, lo, hi, nshift=0, deriv=0, lweight=0):
            kp = torch.as_tensor(np.ascontiguousarray(kprod, dtype=np.float64), device=dev)
            d_r = torch.as_tensor(np.asarray(r_arr, dtype=np.float64), device=dev)
            _lib.call("ps_kint_radial", _vp(table), _vp(d_x), len(x_arr), lmin, nl_tab, _vp(d_k), len(k_arr),
                      _vp(kp), 0 if kp.dim() == 1 else len(k_arr), _vp(d_T), npol, nl_T, _vp(d_r), len(r_arr),
                      lo, hi, nshift, deriv, lweight, npol_out, _vp(out), _stream())
            torch.cuda.current_stream().synchronize()  # kp, d_r are released on return

        if ints_1d:
            assert np.max(x_arr) >= np.max(k_arr) * np.max(self.r_arr)
            if len(self.p_inds) > 0:
                print("Computing p_lL^X(r) integrals")
                plLXs = torch.zeros((2 * self.nmax + 1, lmax + 1, npol_out, self.N_r), dtype=torch.float64,
                                    device=dev)
                for n in range(-max(self.p_inds), max(self.p_inds) + 1):
                    lshift1 = min(0, self.lmin - lmin + n)
                    integral(2. / np.pi * k_arr * k_arr * Pz / 2., self.r_arr, plLXs[self.nmax + n],
                             self.lmin - lshift1, self.lmax, nshift=n)
                self.d_plLXs = plLXs
                self.plLXs = plLXs.cpu().numpy()
            if 'q' in self.to_compute:
                print("Computing q_l^X(r) integrals")
                qlXs = torch.zeros((self.lmax + 1, npol_out, self.N_r), dtype=torch.float64, device=dev)
                integral(2. / np.pi * k_arr * k_arr / 2., self.r_arr, qlXs, self.lmin, self.lmax)
                self.d_qlXs = qlXs
                self.qlXs = qlXs.cpu().numpy()
            if 'r' in self.to_compute:
                print("Computing r_l^X(r) integrals")
                rlXs = torch.zeros((self.lmax + 1, npol_out, self.N_r), dtype=torch.float64, device=dev)
                integral(2. / np.pi * k_arr * k_arr / 2. * Pz ** (3. / 4.), self.r_arr, rlXs, self.lmin, self.lmax)
                self.d_rlXs = rlXs
                self.rlXs = rlXs.cpu().numpy()
        if ints_coll and len(self.coll_params) > 0:
            # p^beta_{lL}^X(r) (collider_p_integral, k_integrals.pyx:399-451): the p sum with the complex
            # kprod = (2/pi) k^(2 + beta) P_zeta / 2 for k >= k_coll, as its real and imaginary parts;
            # beta with Im > 0 follows by conjugation and is not stored
            print("Computing collider p_lL^{beta,X}(r) integrals")
            self.coll_plLXs, self.d_coll_plLXs = {}, {}
            for beta in self.coll_params:
                if np.imag(beta) > 0:
                    continue
                this_nmax = int(np.max(self.coll_params[beta][:, 0]))
                kc = np.where(k_arr >= self.k_coll,
                              2. / np.pi * k_arr.astype(np.complex128) ** (2. + beta) * Pz / 2., 0.)
                parts = []
                for kpart in (kc.real, kc.imag):
                    out = torch.zeros((2 * this_nmax + 1, lmax + 1, npol_out, self.N_r), dtype=torch.float64,
                                      device=dev)
                    for n in range(-this_nmax, this_nmax + 1):
                        lshift1 = min(0, self.lmin - lmin + n)
                        integral(kpart, self.r_arr, out[this_nmax + n], self.lmin - lshift1, self.lmax, nshift=n)
                    parts.append(out)
                d = torch.complex(parts[0], parts[1])
                self.d_coll_plLXs[beta] = d
                self.coll_plLXs[beta] = d.cpu().numpy()
        if ints_2d:
            assert np.max(x_arr) >= np.max(k_arr) * np.max(self.rtau_arr[:, 0])
            r, tau = self.rtau_arr[:, 0], self.rtau_arr[:, 1]
            ktau = k_arr[None, :] * tau[:, None]
            for name, kpow, shape, deriv, lweight, per_r in (('a', 13. / 4., 0, 0, 0, False),
                                                            ('b', 9. / 4., 1, 1, 0, False),
                                                            ('c', 5. / 4., 1, 0, 1, True)):
                if name not in self.to_compute:
                    continue
                print("Computing %s_l^X(r, tau) integrals" % name)
                kpref = 2. / np.pi * k_arr ** kpow * Pz ** (3. / 4.) / 2.
                kp = kpref[None, :] * (np.exp(ktau) if shape == 0 else (1. - ktau) * np.exp(ktau))
                if per_r:
                    kp = kp / r[:, None]
                out = torch.zeros((self.lmax + 1, npol_out, self.N_rtau), dtype=torch.float64, device=dev)
                integral(kp, r, out, self.lmin, self.lmax, deriv=deriv, lweight=lweight)
                setattr(self, 'd_%slXs' % name, out)
                setattr(self, '%slXs' % name, out.cpu().numpy())
        del table
        if ints_1d and len(self.n1n3n) > 0:
            print("Computing F_LL'(r, r') integrals")
            FLLs = torch.zeros((2 * self.nmax_F + 1, self.nLmax + 1, self.N_r, self.N_r), dtype=torch.float64,
                               device=dev)
            pref = 2. * np.pi ** 2 * self.As / self.k_pivot ** (self.ns - 1)
            d_r = torch.as_tensor(np.asarray(self.r_arr, dtype=np.float64), device=dev)
            err = torch.zeros(1, dtype=torch.int32, device=dev)
            _lib.call("ps_tau_F_integral", _vp(d_r), self.N_r, self.Lmin, self.Lmax, self.nmax_F, self.nLmax + 1,
                      float(self.ns), float(pref), _vp(FLLs), _vp(err), _stream())
            if int(err.item()) != 0:
                raise Exception("F_LL'(r, r') calculation failed: a hypergeometric series did not converge")
            self.d_FLLs = FLLs
            self.FLLs = FLLs.cpu().numpy()
        if ints_coll and len(self.coll_params) > 0:
            self._collider_F_integrals()
        self._make_utils()
        print("Precomputation complete")

    def _collider_F_integrals(self):
        """F^beta_{L,L+n}(r, r') of the collider templates (polyspec/tspec_template.py:670-703 with
        compute_collider_F_integral, k_integrals.pyx:496-545): j_L on the reference's y grid
        (ps_kint_bessel_table), interpolated to 5000 log-spaced K <= 1.01 K_coll (ps_kint_collider_jlK),
        then the trapezium rule over K with (2/pi) K^(2 - 2 beta) P_zeta(K) / 2 (ps_kint_collider_F)."""
        dev = self._dev
        K_arr = np.geomspace(0.1 / (self.r_hor + 5000), self.K_coll * 1.01, 5000)
        this_Lmax = self.Lmax + self.nmax_coll_F
        this_Lmin = max([self.Lmin - self.nmax_coll_F, 0])
        max_Kr = self.K_coll * np.max(self.r_arr)
        y_arr = np.asarray(list(np.arange(0, this_Lmax * 2, 0.01)) + list(np.arange(this_Lmax * 2, max_Kr * 1.01,
                                                                                     0.01)), dtype=np.float64)
        d_y = torch.as_tensor(y_arr, device=dev)
        nl = this_Lmax - this_Lmin + 1
        table = torch.empty((nl, len(y_arr)), dtype=torch.float64, device=dev)
        _lib.call("ps_kint_bessel_table", _vp(d_y), len(y_arr), this_Lmin, this_Lmax, _vp(table), _stream())
        if not bool(torch.isfinite(table).all()):
            raise Exception("Spherical Bessel calculation failed!")
        d_K = torch.as_tensor(K_arr, device=dev)
        d_r = torch.as_tensor(np.asarray(self.r_arr, dtype=np.float64), device=dev)
        jlK = torch.empty((nl, len(K_arr), self.N_r), dtype=torch.float64, device=dev)
        _lib.call("ps_kint_collider_jlK", _vp(table), _vp(d_y), len(y_arr), nl, _vp(d_K), len(K_arr), _vp(d_r),
                  self.N_r, _vp(jlK), _stream())
        del table
        print("Computing F_LL'^beta(r, r') integrals")
        self.coll_FLLs, self.d_coll_FLLs = {}, {}
        nLout = self.base.lmax + 1
        for beta in self.coll_params:
            if np.imag(beta) > 0:
                continue
            this_nmax_F = int(np.max(self.coll_params[beta][:, 1]))
            Kprod = np.where(K_arr <= self.K_coll,
                             2. / np.pi * K_arr.astype(np.complex128) ** (2. - 2. * beta) * self.Pzeta(K_arr) / 2., 0.)
            d_Kp = torch.as_tensor(Kprod.astype(np.complex128), device=dev)
            F = torch.zeros((2 * this_nmax_F + 1, nLout, self.N_r, self.N_r), dtype=torch.complex128, device=dev)
            _lib.call("ps_kint_collider_F", _vp(jlK), nl, this_Lmin, _vp(d_K), len(K_arr), _vp(d_Kp), self.N_r,
                      self.Lmin, self.Lmax, this_nmax_F, nLout, _vp(F), _stream())
            torch.cuda.current_stream().synchronize()
            self.d_coll_FLLs[beta] = F
            self.coll_FLLs[beta] = F.cpu().numpy()
        del jlK

    def set_radial_integrals(self, qlXs=None, plLXs=None, **arrays):
        """Install precomputed radial integrals in place of the computed ones: any of
        qlXs, rlXs [lmax+1, 1+2 pol, N_r], plLXs [2 nmax+1, lmax+2, 1+2 pol, N_r], alXs,
        blXs, clXs [lmax+1, 1+2 pol, N_rtau] (the reference's attribute names and layouts)."""
        arrays.update(qlXs=qlXs, plLXs=plLXs)
        if arrays.get('FLLs') is not None:
            arrays['FLLs'] = np.ascontiguousarray(arrays['FLLs'], dtype=np.float64)
        for name, arr in arrays.items():
            if arr is None:
                continue
            a = np.asarray(arr, dtype=np.float64)
            setattr(self, name, a)
            setattr(self, 'd_' + name, torch.as_tensor(a, device=self._dev))

    def _make_utils(self):
        self.utils = pixel.tauNL_utils(self.base.nthreads, self.N_r, self.base.l_arr.astype(np.int32),
                                       self.base.m_arr.astype(np.int32), self.Lmin, self.Lmax,
                                       self.ls.astype(np.int32), self.ms.astype(np.int32),
                                       self.Ls.astype(np.int32), self.Ms.astype(np.int32), self.nmax_F)
        self.d_nLminfilt_idx = torch.as_tensor(np.nonzero(self.nLminfilt)[0], device=self._dev)
        if len(self.n1n3n) > 0:
            # per lm of the l <= nLmax list: L where Lmin <= L <= Lmax (else -1), and the m weight
            sel = self.base.l_arr <= self.nLmax
            L, M = self.base.l_arr[sel], self.base.m_arr[sel]
            lm_L = np.where((L >= self.Lmin) & (L <= self.Lmax), L, -1).astype(np.int32)
            self.d_tau_lm_L = torch.as_tensor(lm_L, device=self._dev)
            self.d_tau_lm_w = torch.as_tensor(np.where(M == 0, 1., 2.), device=self._dev)
            self.d_r_weights = {t: torch.as_tensor(np.asarray(self.r_weights[t], dtype=np.float64), device=self._dev)
                                for t in self.templates if t in self.r_weights}

    # ------------------------------------------------------------------ timings
    def report_timings(self):
        """Timers (polyspec/tspec_template.py:453-497)."""
        print("\n## Timings ##\n")
        print("Precomputation: %.2fs" % self.timers['precomputation'])
        for k, name in (('numerator', 'Numerator'), ('fisher', 'Fisher'), ('optimization', 'Optimization')):
            if self.timers[k] != 0:
                print("%s: %.2fs" % (name, self.timers[k]))
        print("\n# Timing Breakdown")
        if self.timers['Sinv'] != 0:
            print("S^-1 filtering: %.2fs" % self.timers['Sinv'])
        if self.timers['map_transforms'] != 0:
            print("1-field transforms: %.2fs" % self.timers['map_transforms'])
        if self.timers['numerator'] != 0:
            if np.any([('gNL' in t) for t in self.templates]):
                print("gNL -- 4-field summation: %.2fs" % self.timers['gNL_summation'])
            if 'lensing' in self.templates:
                print("Lensing -- 2-field transforms: %.2fs" % self.timers['lensing_products'])
                print("Lensing -- 4-field summation: %.2fs" % self.timers['lensing_summation'])
        if self.timers['fisher'] != 0:
            if self.timers['fish_grfs'] != 0:
                print("Fisher -- creating GRFs: %.2fs" % self.timers['fish_grfs'])
            if self.timers['Ainv'] != 0:
                print("Fisher -- A^-1 filtering: %.2fs" % self.timers['Ainv'])
            print("Fisher -- 3-field derivatives: %.2fs" % self.timers['fish_deriv'])
            print("Outer product: %.2fs" % self.timers['fish_outer'])
        print("\n## Harmonic Transforms ##")
        print("Forward: %d" % self.base.n_SHTs_forward)
        print("Reverse: %d" % self.base.n_SHTs_reverse)
        print("Time: %.2fs" % self.base.time_sht)
        print("\n")

    def reset_timings(self):
        for f in self.timers.keys():
            self.timers[f] = 0.
        self.base.n_SHTs_forward = 0
        self.base.n_SHTs_reverse = 0
        self.base.time_sht = 0.

    def _timed(self, key, t0):
        torch.cuda.current_stream().synchronize()
        self.timers[key] += time.time() - t0

    # ------------------------------------------------------------------ filtered maps
    def _full_lm(self, h_filt, lmax):
        """Embed [..., nlm(l in [lmin, lmax])] into the full [..., nlm(lmax)] layout (zeros below lmin)."""
        n = (lmax + 1) * (lmax + 2) // 2
        out = torch.zeros(h_filt.shape[:-1] + (n,), dtype=torch.complex128, device=h_filt.device)
        out[..., self.d_lminfilt] = h_filt
        return out

    def _compute_weighted_maps(self, h_lm_filt, flX_arr, spin=0):
        """[Sum_lm {}_sY_lm(i) f_l^X(i) h_lm] maps for each sampling point (polyspec/tspec_template.py:799-815);
        for spin 1 the (+1) maps of the spin-1 transform of [-summ, 0]."""
        t0 = time.time()
        summ = self._full_lm(self.utils.apply_fl_weights(flX_arr, h_lm_filt, 1.), self.lmax)
        out = self.base.to_map_vec(summ, output_spin=spin, lmax=self.lmax)
        if spin != 0:
            out = out[0]
        self._timed('map_transforms', t0)
        return out

    def _compute_weighted_gaunt_maps(self, h_lm_filt, flLX_arr_re, n, mu, flLX_arr_im=None):
        """P_{n,mu} maps [N_r, Npix] of polyspec/tspec_template.py:817-876:
        n = 0 is the transfer-weighted synthesis of h / sqrt(4 pi); n > 0 sums the Gaunt-weighted
        shifts l -> l + Delta of conj(h) (``shift_and_weight_map_all``) into real- and imaginary-part
        harmonics up to lmax + n and combines their syntheses as re - i im (complex maps).  With the
        imaginary part of complex (collider) integrals, n = 0 gives the complex map R + i I and n > 0
        adds the i-weighted shifts of the imaginary part with the two outputs exchanged."""
        assert mu <= n, "mu<=n is required!"
        assert mu >= 0, "Negative mu can be obtained by conjugation properties"
        t0 = time.time()
        nmax = len(flLX_arr_re) // 2
        if n == 0:
            summ = self._full_lm(self.utils.apply_fl_weights(flLX_arr_re[nmax], h_lm_filt,
                                                             1. / np.sqrt(4. * np.pi)), self.lmax)
            out = self.base.to_map_vec(summ, lmax=self.lmax)
            if flLX_arr_im is not None:
                summ = self._full_lm(self.utils.apply_fl_weights(flLX_arr_im[nmax], h_lm_filt,
                                                                 1. / np.sqrt(4. * np.pi)), self.lmax)
                out = pixel.r2c(out, self.base.to_map_vec(summ, lmax=self.lmax))
        else:
            nr = flLX_arr_re.shape[3]
            nt = int(np.sum(self.base.l_arr <= self.lmax + n))
            Lr = torch.zeros((nr, nt), dtype=torch.complex128, device=self._dev)
            Li = torch.zeros_like(Lr)
            self.utils.shift_and_weight_map_all(flLX_arr_re, h_lm_filt, n, mu, 1.0, Lr, Li, nmax)
            if flLX_arr_im is not None:
                self.utils.shift_and_weight_map_all(flLX_arr_im, h_lm_filt, n, mu, 1.0j, Li, Lr, nmax)
            if bool((Li.imag != 0.).any()):
                out = pixel.r2cstar(self.base.to_map_vec(Lr, lmax=self.lmax + n),
                                    self.base.to_map_vec(1.0j * Li, lmax=self.lmax + n))
            else:
                out = self.base.to_map_vec(Lr, lmax=self.lmax + n)
        self._timed('map_transforms', t0)
        return out

    def _compute_lensing_U_map(self, h_lm_filt):
        """[U^T, U^E, U^B] (polyspec/tspec_template.py:878-910)."""
        t0 = time.time()
        b = self.base
        U = torch.zeros((1 + 2 * self.pol, b.Npix), dtype=torch.complex128, device=self._dev)
        inp = self._full_lm(h_lm_filt[0], self.lmax)
        U[0] = b.to_map(inp[None], lmax=self.lmax)[0]
        if 'lensing' in self.templates and self.pol:
            for X in (1, 2):
                inp = self._full_lm(h_lm_filt[X], self.lmax)
                U[X] = b.to_map_spin(inp, inp, spin=2, lmax=self.lmax)[0]
        self._timed('map_transforms', t0)
        return U

    def _compute_lensing_V_map(self, h_lm_filt):
        """[V^T, V^{E,B}(+), V^{E,B}(-)] (polyspec/tspec_template.py:912-965)."""
        t0 = time.time()
        b = self.base
        ls = torch.as_tensor(self.ls.astype(np.float64), device=self._dev)
        lsi = torch.as_tensor(self.ls, device=self._dev)
        C = {k: torch.as_tensor(np.asarray(v, dtype=np.float64), device=self._dev)[lsi]
             for k, v in self.C_lens_weight.items()}
        V = torch.zeros((1 + 2 * self.pol, b.Npix), dtype=torch.complex128, device=self._dev)
        if not self.pol:
            inp = self._full_lm(torch.sqrt(ls * (ls + 1.)) * C['TT'] * h_lm_filt[0], self.lmax)
            V[0] = b.to_map_spin(-inp, inp, spin=1, lmax=self.lmax)[1]
        else:
            wienerT = C['TT'] * h_lm_filt[0] + C['TE'] * h_lm_filt[1]
            inp = self._full_lm(torch.sqrt(ls * (ls + 1.)) * wienerT, self.lmax)
            V[0] = b.to_map_spin(-inp, inp, spin=1, lmax=self.lmax)[1]
            pref_p = torch.sqrt((ls + 2.) * (ls - 1.))
            pref_m = torch.sqrt((ls - 2.) * (ls + 3.))
            wienerE = C['TE'] * h_lm_filt[0] + C['EE'] * h_lm_filt[1]
            wienerB = C['BB'] * h_lm_filt[2]
            re = self._full_lm(pref_p * wienerE, self.lmax)
            im = self._full_lm(1.0j * pref_p * wienerB, self.lmax)
            V[1] = b.to_map_spin(re + im, -re + im, spin=1, lmax=self.lmax)[0]
            re = self._full_lm(pref_m * wienerE, self.lmax)
            im = self._full_lm(1.0j * pref_m * wienerB, self.lmax)
            V[2] = b.to_map_spin(re + im, -re + im, spin=3, lmax=self.lmax)[0]
        self._timed('map_transforms', t0)
        return V

    def _apply_all_filters(self, input_map):
        """Filtered maps of one S^-1-weighted field (polyspec/tspec_template.py:1036-1096)."""
        output = {}
        if 'a' in self.to_compute:
            output['a'] = self._compute_weighted_maps(input_map, self.d_alXs)
        if 'b' in self.to_compute:
            output['b'] = self._compute_weighted_maps(input_map, self.d_blXs)
        if 'c' in self.to_compute:
            output['c'] = self._compute_weighted_maps(input_map, self.d_clXs, spin=1)
        for n in self.p_inds:
            for mu in range(n + 1):
                output['p%d%d' % (n, mu)] = self._compute_weighted_gaunt_maps(input_map, self.d_plLXs, n, mu)
        for beta in self.coll_params:
            # collider P^beta_{s,lam} maps (polyspec/tspec_template.py:1058-1089); Im beta > 0 from the conjugate
            if np.imag(beta) != 0:
                if np.imag(beta) <= 0:
                    P = self.d_coll_plLXs[beta]
                    re, im = P.real.contiguous(), P.imag.contiguous()
                else:
                    P = self.d_coll_plLXs[np.conj(beta)]
                    re, im = P.real.contiguous(), (-P.imag).contiguous()
            else:
                re, im = self.d_coll_plLXs[beta].real.contiguous(), None
            maps = {}
            for s_ in np.unique(self.coll_params[beta][:, 0]):
                for lam in range(int(s_) + 1):
                    maps['p%d%d' % (s_, lam)] = self._compute_weighted_gaunt_maps(input_map, re, int(s_), lam, im)
            output[_ckey(beta)] = maps
        if 'q' in self.to_compute:
            output['q'] = self._compute_weighted_maps(input_map, self.d_qlXs)
        if 'r' in self.to_compute:
            output['r'] = self._compute_weighted_maps(input_map, self.d_rlXs)
        if 'u' in self.to_compute:
            output['u'] = self._compute_lensing_U_map(input_map)
        if 'v' in self.to_compute:
            output['v'] = self._compute_lensing_V_map(input_map)
        return output

    def _filter_pair(self, input_maps, filtering='Q'):
        """Filtered fields of a pair of inputs (polyspec/tspec_template.py:967-1034)."""
        if filtering == 'P':
            out = {}
            for n in self.p_inds:
                out[n] = torch.stack([torch.stack([self._compute_weighted_gaunt_maps(m, self.d_plLXs, n, mu)
                                                   for mu in range(n + 1)]) for m in input_maps])
            return out
        if filtering == 'coll-P':
            # collider P^beta_{s,lam} maps [2, s+1, N_r, Npix] per (beta, s) (polyspec/tspec_template.py:995-1019)
            out = {}
            for beta in self.coll_params:
                if np.imag(beta) == 0:
                    re, im = self.d_coll_plLXs[beta].real.contiguous(), None
                elif np.imag(beta) < 0:
                    re, im = self.d_coll_plLXs[beta].real.contiguous(), self.d_coll_plLXs[beta].imag.contiguous()
                else:
                    P = self.d_coll_plLXs[np.conj(beta)]
                    re, im = P.real.contiguous(), (-P.imag).contiguous()
                for s_ in np.unique(self.coll_params[beta][:, 0]):
                    s_ = int(s_)
                    out[beta, s_] = torch.stack([torch.stack([
                        self._compute_weighted_gaunt_maps(m, re, s_, lam, im).to(torch.complex128)
                        for lam in range(s_ + 1)]) for m in input_maps])
            return out
        spin0 = {'Q': 'd_qlXs', 'R': 'd_rlXs', 'A': 'd_alXs', 'B': 'd_blXs'}
        if filtering in spin0:
            return torch.stack([self._compute_weighted_maps(m, getattr(self, spin0[filtering])) for m in input_maps])
        if filtering == 'C':
            return torch.stack([self._compute_weighted_maps(m, self.d_clXs, spin=1) for m in input_maps])
        if filtering == 'U':
            return torch.stack([self._compute_lensing_U_map(m) for m in input_maps])
        if filtering == 'V':
            return torch.stack([self._compute_lensing_V_map(m) for m in input_maps])
        raise Exception("Filtering %s is not implemented!" % filtering)

    def _compute_lensing_Phi(self, maps1, maps2, add_sym=False):
        """Phi_LM of the lensing estimators (polyspec/tspec_template.py:1098-1108)."""
        t0 = time.time()
        if add_sym:
            inp = pixel.lens_phi_sum_sym(maps1['u'], maps2['u'], maps1['v'], maps2['v'])
        else:
            inp = pixel.lens_phi_sum(maps1['u'], maps2['v'])
        pm = self.base.to_lm_spin(inp, inp.conj(), spin=1, lmax=self.Lmax_lens)
        out = (-0.25 * (pm[0] - pm[1]))[self.d_Lminfilt_lens]
        self._timed('lensing_products', t0)
        return out

    def _lens_Ls(self):
        filt = (self.base.l_arr >= self.Lmin_lens) * (self.base.l_arr <= self.Lmax_lens)
        Ls = self.base.l_arr[filt]
        Ms = self.base.m_arr[filt]
        w = Ls * (Ls + 1.) * (1. + (Ms > 0)) * np.asarray(self.C_phi)[Ls]
        return torch.as_tensor(w, device=self._dev)

    def _check_sampling(self):
        if self.ints_1d and (not hasattr(self, 'r_arr')):
            raise Exception("Need to supply radial integration points or run optimize_radial_sampling_1d()!")
        if self.ints_2d and (not hasattr(self, 'rtau_arr')):
            raise Exception("Need to supply radial/tau integration points or run optimize_radial_sampling_2d()!")

    # ------------------------------------------------------------------ simulations
    def _sinv_filt(self, x, input_type='map'):
        y = self.applySinv(x, input_type=input_type, lmax=self.lmax)
        return y[:, self.d_lminfilt].contiguous()

    def _process_sim(self, sim_pair, input_type='map'):
        """Filtered maps of one simulation pair (polyspec/tspec_template.py:1110-1126)."""
        t0 = time.time()
        dt = torch.float64 if input_type == 'map' else torch.complex128
        ha = self._sinv_filt(self.base._in(sim_pair[0], dt)[0], input_type)
        hb = self._sinv_filt(self.base._in(sim_pair[1], dt)[0], input_type)
        self._timed('Sinv', t0)
        return self._apply_all_filters(ha), self._apply_all_filters(hb)

    def load_sims(self, load_sim_pair, N_pairs, verb=False, preload=True, input_type='map'):
        """Simulation pairs for the disconnected terms (polyspec/tspec_template.py:1128-1170)."""
        self.N_it = N_pairs
        print("Using %d pairs of Monte Carlo simulations" % self.N_it)
        if preload:
            self.preload = True
            self._check_sampling()
            self.proc_a_maps, self.proc_b_maps = [], []
            for ii in range(self.N_it):
                if ii % 5 == 0 and verb:
                    print("Processing bias simulation pair %d of %d" % (ii + 1, self.N_it))
                a, b = self._process_sim(load_sim_pair(ii), input_type=input_type)
                self.proc_a_maps.append(a)
                self.proc_b_maps.append(b)
        else:
            self.preload = False
            if verb:
                print("No preloading; simulations will be loaded and accessed at runtime.")
            self.load_sim_data = lambda ii: self._process_sim(load_sim_pair(ii), input_type=input_type)

    def generate_sims(self, N_pairs, Cl_input=[], preload=True, verb=False):
        """GRF simulation pairs for the disconnected terms (polyspec/tspec_template.py:1172-1229)."""
        self.N_it = N_pairs
        print("Using %d pairs of Monte Carlo simulations" % self.N_it)
        if len(Cl_input) == 0:
            Cl_input = self.base.Cl_tot
        b = self.base

        def pair(ii):
            if self.ones_mask:
                alpha = b.generate_data(int(1e5) + ii, Cl_input=Cl_input, output_type='harmonic', lmax=self.lmax,
                                        deconvolve_beam=False)
                beta = b.generate_data(int(2e5) + ii, Cl_input=Cl_input, output_type='harmonic', lmax=self.lmax,
                                       deconvolve_beam=False)
                return self._process_sim([alpha, beta], input_type='harmonic')
            alpha = self.d_mask * b._in(b.generate_data(int(1e5) + ii, Cl_input=Cl_input, deconvolve_beam=False),
                                        torch.float64)[0]
            beta = self.d_mask * b._in(b.generate_data(int(2e5) + ii, Cl_input=Cl_input, deconvolve_beam=False),
                                       torch.float64)[0]
            return self._process_sim([alpha, beta])

        if preload:
            self.preload = True
            self._check_sampling()
            self.proc_a_maps, self.proc_b_maps = [], []
            for ii in range(self.N_it):
                if ii % 5 == 0 and verb:
                    print("Generating bias simulation pair %d of %d" % (ii + 1, self.N_it))
                a, bb = pair(ii)
                self.proc_a_maps.append(a)
                self.proc_b_maps.append(bb)
        else:
            self.preload = False
            if verb:
                print("No preloading; simulations will be loaded and accessed at runtime.")
            self.load_sim_data = pair

    # ------------------------------------------------------------------ local tauNL
    def _decompose_tauNL_even(self, n):
        """(n1, n3, n) pieces of tauNL-even:n and their weights (polyspec/tspec_template.py:754-760)."""
        pref = (-1.) ** n / 3. * (4. * np.pi) ** 1.5 / np.sqrt(2. * n + 1.)
        if n == 0:
            return [[0, 0, 0]], [3 * pref]
        return [[n, n, 0], [0, n, n]], [pref, 2 * pref]

    def _decompose_tauNL_odd(self, n):
        """(n1, n3, n) pieces of tauNL-odd:n and their weights (polyspec/tspec_template.py:762-796): for N, N' in
        |n-1|..n+1, weight (-1)^n sqrt(2)/3 (4 pi)^(3/2) sqrt((2N+1)(2N'+1)) (N 1 n; 0 0 0)(N' 1 n; 0 0 0)
        {N 1 N'; 1 n 1} on (min, max, 1) (with (-1)^(N+N') when N > N') and, times 1 + (-1)^(n+N+1), on
        (1, N, N'); equal pieces summed, in sorted order."""
        pref = (-1.) ** n * np.sqrt(2.) / 3. * (4. * np.pi) ** 1.5
        parts, weights = [], []
        for N in range(abs(n - 1), n + 2):
            f1 = wig3zero(N, 1, n)
            if f1 == 0:
                continue
            for Np in range(abs(n - 1), n + 2):
                f12 = f1 * wig3zero(Np, 1, n)
                if f12 == 0:
                    continue
                f12 *= wig6(N, 1, Np, 1, n, 1)
                if f12 == 0:
                    continue
                w = pref * np.sqrt(2. * N + 1.) * np.sqrt(2. * Np + 1.) * f12
                if Np >= N:
                    parts.append([N, Np, 1])
                    weights.append(w)
                else:
                    parts.append([Np, N, 1])
                    weights.append((-1) ** (Np + N) * w)
                parts.append([1, N, Np])
                weights.append(w * (1. + (-1) ** (n + N + 1)))
        uniq = [list(u) for u in np.unique(parts, axis=0)] if parts else []
        return uniq, [float(np.sum([weights[i] for i in range(len(parts)) if parts[i] == u])) for u in uniq]

    def _direc_parts(self, t):
        """[(n1, n3, n, weight)] of a direction-dependent template: tauNL-direc:n1,n3,n alone, or the
        decomposition of tauNL-even:n / tauNL-odd:n.  Its 4-, 2- and 0-field numerator terms and its Fisher
        derivative are the weighted sums of the tauNL-direc ones (polyspec/tspec_template.py:1433-1487,
        :1689-1815, :2850-2893)."""
        if 'tauNL-direc' in t:
            n1, n3, n = (int(x) for x in t.split(':')[1].split(','))
            return [(n1, n3, n, 1.)]
        n = int(t.split(':')[1])
        parts, weights = (self._decompose_tauNL_even(n) if 'tauNL-even' in t else self._decompose_tauNL_odd(n))
        return [(int(a), int(b), int(c), float(w)) for (a, b, c), w in zip(parts, weights)]

    def _A_maps(self, map1, map2, n, add_sym=False, beta=None):
        """[P_{n,mu} Q]_LM for mu = -n..n and each radial sample (polyspec/tspec_template.py:1275-1334), as
        [2n+1, N_r, nlm(nLmax)] over the full l <= nLmax list (entries with L < nLmin are unused);
        optionally adding the map1 <-> map2 term.  mu < 0 uses conjugation, (-1)^(n+mu) conj(P_{n,-mu}).
        With a collider beta the P maps are the P^beta_{n,mu} (complex for complex beta; mu < 0 then
        conjugates the maps of conj(beta))."""
        t0 = time.time()

        def P(mp, key):
            return mp[key] if beta is None else mp[_ckey(beta)][key]

        def Pc(mp, key):
            return mp[key] if beta is None else mp[_ckey(np.conj(beta) if np.imag(beta) != 0 else beta)][key]

        if n == 0:
            if beta is None or np.imag(beta) == 0:
                if add_sym:
                    prod = pixel.multiplyRR_sym(map2['q'], P(map1, 'p00'), map1['q'], P(map2, 'p00'))
                else:
                    prod = pixel.multiplyRR(map2['q'], P(map1, 'p00'))
                out = self.base.to_lm_vec(prod, lmax=self.nLmax)[None]
            else:
                if add_sym:
                    prod = pixel.multiplyRC_sym(map2['q'], P(map1, 'p00'), map1['q'], P(map2, 'p00'))
                else:
                    prod = pixel.multiplyRC(map2['q'], P(map1, 'p00'))
                out = self.base.to_lm_vec(prod.real.contiguous(), lmax=self.nLmax).to(torch.complex128)
                if bool((prod.imag[:, 0] != 0).any()):
                    out = out + 1j * self.base.to_lm_vec(prod.imag.contiguous(), lmax=self.nLmax)
                out = out[None]
            self._timed('tauNL_summation', t0)
            return out
        output = []
        for mu in range(-n, n + 1):
            key = 'p%d%d' % (n, abs(mu))
            if mu < 0:
                fac = (-1.) ** (n + mu)
                if add_sym:
                    prod = pixel.multiplyRCstar_sym(map2['q'], Pc(map1, key), map1['q'], Pc(map2, key), fac)
                else:
                    prod = pixel.multiplyRCstar(map2['q'], Pc(map1, key), fac)
            else:
                if add_sym:
                    prod = pixel.multiplyRC_sym(map2['q'], P(map1, key), map1['q'], P(map2, key))
                else:
                    prod = pixel.multiplyRC(map2['q'], P(map1, key))
            out = self.base.to_lm_vec(prod.real.contiguous(), lmax=self.nLmax).to(torch.complex128)
            if bool((prod[:, 0].imag != 0).any()):
                out = out + 1j * self.base.to_lm_vec(prod.imag.contiguous(), lmax=self.nLmax)
            output.append(out)
        self._timed('tauNL_summation', t0)
        return torch.stack(output)

    def _tau_convolve(self, X, weights, A=None):
        """pixel.tau_convolve_F over [N_r, nlm(nLmax)] harmonic maps: the F_L convolution of X
        (polyspec/cython/tauNL_utils.pyx:966-995) or, with A, the tau sum of (A, X) (:604-647)."""
        return pixel.tau_convolve_F(X, self.d_tau_lm_L, self.d_FLLs[self.nmax_F], weights, A=A,
                                    lm_w=self.d_tau_lm_w)

    def _tau_sum(self, A, B, weights, n1, n3, n):
        """Sum over mu1, mu3, mu, (L, M), (L', M'), (r, r') of the tauNL estimators
        (polyspec/tspec_template.py:1231-1240).  n = 0 (n1 = n3): Sum_mu tau(A[n1][mu], B[n1][mu]) / sqrt(2 n1 + 1)
        (tauNL_utils.pyx:604-647); n > 0: the Gaunt- and 3j-weighted sum of tauNL_utils.pyx:650-715 over the
        A[n1], B[n3] maps in the reference's [2n+1, len(Ls), N_r] layout."""
        t0 = time.time()
        if n == 0:
            assert n1 == n3
            out = 0.
            for mu in range(A[n1].shape[0]):
                out += self._tau_convolve(B[n1][mu], weights, A=A[n1][mu])
            out /= np.sqrt(2. * n1 + 1.)
        else:
            def rows(X):
                return X[:, :, self.d_nLminfilt_idx].permute(0, 2, 1).contiguous()
            out = self.utils.tau_sum_general(rows(A[n1]), rows(B[n3]), self.d_FLLs, weights, n1, n3, n)
        self._timed('tauNL_summation', t0)
        return out

    def _calC(self, s, S, mu_s):
        """C_s(S, mu_s) coupling of the collider templates (polyspec/tspec_template.py:710-743): for mu_s = 0,
        delta_S0 (4 pi)^(3/2) (-1)^s / sqrt(2s+1); otherwise (4 pi)^(3/2) sqrt(2S+1)/(2s+1) Sum_lam (-1)^(S+lam)
        W_lam(s, mu_s) (s s S; lam -lam 0), W_lam = G(1/2+s-i mu) G(1/2+lam+i mu) / (G(1/2+s+i mu) G(1/2+lam-i mu))."""
        from scipy.special import gamma

        def W_lam(lam, s, mu_s):
            assert abs(lam) <= s
            if np.real(mu_s) == 0.:
                mu_s += 1e-12
            W = gamma(0.5 + s - 1.0j * mu_s) * gamma(0.5 + lam + 1.0j * mu_s) / (
                gamma(0.5 + s + 1.0j * mu_s) * gamma(0.5 + lam - 1.0j * mu_s))
            return W.real if np.real(mu_s) == 1e-12 else W

        if s == 0 and np.real(mu_s) == 0:
            nu_s = np.real(-1.0j * mu_s)
            assert 0. <= nu_s <= 1.5, "Light spin-0 particles have nu_s in (0, 3/2)"
        elif np.real(mu_s) == 0:
            nu_s = np.real(-1.0j * mu_s)
            assert 0 <= nu_s <= s - 0.5, "Light spin-%d particles have nu_s in (0, %.1f)" % (s, s - 1. / 2.)
            assert nu_s <= 0.5, "Couplings undefined for Higuchi-bound violating particles!"
        else:
            assert np.imag(mu_s) == 0, "mu_s can't be complex!"
        if mu_s == 0.:
            return (S == 0) * (4. * np.pi) ** (3. / 2.) / np.sqrt(2. * s + 1.) * (-1.) ** s
        pref = (4. * np.pi) ** (3. / 2.) / (2. * s + 1.) * np.sqrt(2. * S + 1.)
        out = 0.
        for lam in range(-s, s + 1):
            out += (-1.) ** (S + lam) * W_lam(lam, s, mu_s) * wig3(s, s, S, lam, -lam, 0)
        return np.real_if_close(pref * out)

    def _omega_prime(self, s, mu_s):
        """S-independent phase omega'_s(mu_s) of the collider coupling (polyspec/tspec_template.py:744-754):
        zero for light particles, else arg(-2^(-4 i mu) (1 + i sinh(pi mu)) (5/2 + s + i mu)^2 /
        (3/2 + s - i mu)^2 G(-i mu)^2 G(1/2 + s + i mu)^2)."""
        from scipy.special import gamma
        if np.real(mu_s) == 0:
            return 0.
        val = 2. ** (-4. * mu_s * 1.0j) * (1. + 1.0j * np.sinh(np.pi * mu_s)) * (2.5 + s + 1.0j * mu_s) ** 2. \
            / (1.5 + s - 1.0j * mu_s) ** 2.
        val *= gamma(-1.0j * mu_s) ** 2 * gamma(0.5 + s + 1.0j * mu_s) ** 2
        return np.angle(-1. * val)

    def _coll_rows(self, X):
        """[2s+1, N_r, nlm(nLmax)] harmonic maps -> the reference's [2s+1, len(Ls), N_r] row layout."""
        return X[:, :, self.d_nLminfilt_idx].permute(0, 2, 1).contiguous()

    def _tau_sum_collider(self, A, B, weights, s, beta):
        """Sum over lam1, lam3, Lam, S, (L, M), (L', M'), (r, r') of the collider estimator
        (polyspec/tspec_template.py:1243-1273): s = 0 and nu_s = 0 take the diagonal forms
        (ps_tau_sum_collider_diag), otherwise the general Gaunt/3j sum (ps_tau_sum_collider_general)."""
        t0 = time.time()
        pos = _ckey_s(s, beta)
        neg = pos if np.imag(beta) == 0 else _ckey_s(s, np.conj(beta))
        nu_s = beta + 3. / 2.
        nF = int(np.max(self.coll_params[beta][:, 1]))
        F = self.d_coll_FLLs[beta]
        w = np.asarray(weights, dtype=np.float64)
        if s == 0:
            tau = self.utils.tau_sum_n0_collider(self._coll_rows(A[pos]), self._coll_rows(B[neg]), F[nF], w,
                                                 4. * np.pi * np.exp(1.0j * self._omega_prime(0, 1.0j * nu_s)))
        elif nu_s == 0:
            tau = self.utils.tau_sum_nu0_collider(self._coll_rows(A[pos]), self._coll_rows(B[neg]), F[nF], w,
                                                  4. * np.pi / (2. * s + 1.) * (-1.) ** s)
        else:
            coeffs = np.asarray([np.exp(1.0j * self._omega_prime(s, 1.0j * nu_s)) * self._calC(s, S, 1.0j * nu_s)
                                 for S in range(0, 2 * s + 1, 2)], dtype=np.complex128)
            tau = self.utils.tau_sum_general_collider(self._coll_rows(A[pos]), self._coll_rows(A[neg]),
                                                      self._coll_rows(B[pos]), self._coll_rows(B[neg]), F, w, nF, s,
                                                      beta, coeffs)
        self._timed('tauNL_summation', t0)
        return tau

    def set_collider_integrals(self, coll_plLXs=None, coll_FLLs=None):
        """Install precomputed collider integrals (dicts beta -> the reference's coll_plLXs
        [2 nmax+1, lmax+2, 1+2 pol, N_r] and coll_FLLs [2 nmax_F+1, lmax+1, N_r, N_r], complex) in place of
        the computed ones."""
        for name, arrs in (('coll_plLXs', coll_plLXs), ('coll_FLLs', coll_FLLs)):
            if arrs is None:
                continue
            host = {k: np.asarray(v, dtype=np.complex128) for k, v in arrs.items()}
            setattr(self, name, host)
            setattr(self, 'd_' + name, {k: torch.as_tensor(v, device=self._dev) for k, v in host.items()})

    def _coll_lm(self, x):
        """Harmonic rows [len(Ls), N_r] of maps [N_r, Npix] up to nLmax."""
        return self.base.to_lm_vec(x.contiguous(), lmax=self.nLmax)[:, self.d_nLminfilt_idx].T

    def _compute_coll_PQ_vecs(self, Ps_maps, Q_maps, i, j, s, beta, add_sym=False, conjPs_maps=None):
        """[P^beta_{s,lam} Q]_LM vectors [2s+1, len(Ls), N_r] of polyspec/tspec_template.py:2012-2137, and for complex
        beta those of the conjugate maps."""
        def prod(P1, P2, lam, fac=None):
            if fac is None:
                if add_sym:
                    return pixel.multiplyRC_sym(Q_maps[j], P1[i, lam], Q_maps[i], P2[j, lam])
                return pixel.multiplyRC(Q_maps[j], P1[i, lam])
            if add_sym:
                return pixel.multiplyRCstar_sym(Q_maps[j], P1[i, lam], Q_maps[i], P2[j, lam], fac)
            return pixel.multiplyRCstar(Q_maps[j], P1[i, lam], fac)

        if s == 0:  # with complex beta the conjugate vector is a - i b of the same product (the reference's :2016-2033)
            pm = prod(Ps_maps, Ps_maps, 0)
            if np.imag(beta) == 0:
                return self._coll_lm(pm.real)[None]
            a, b = self._coll_lm(pm.real), self._coll_lm(pm.imag)
            return (a + 1j * b)[None], (a - 1j * b)[None]
        nrow = int(np.sum(self.nLminfilt))
        nr = Q_maps.shape[1]
        PQ = torch.zeros((2 * s + 1, nrow, nr), dtype=torch.complex128, device=self._dev)
        if conjPs_maps is None:
            assert np.imag(beta) == 0.
            for lam3 in range(s + 1):
                pm = prod(Ps_maps, Ps_maps, lam3)
                if lam3 == 0 and s % 2 == 0:
                    PQ[s] = self._coll_lm(pm.real)
                elif lam3 == 0:
                    PQ[s] = 1.0j * self._coll_lm(pm.imag)
                else:
                    pr, pi = self._coll_lm(pm.real), 1.0j * self._coll_lm(pm.imag)
                    PQ[s + lam3] = pr + pi
                    PQ[s - lam3] = (-1.) ** (s - lam3) * (pr - pi)
            return PQ
        cPQ = torch.zeros_like(PQ)
        for lam3 in range(-s, s + 1):
            if lam3 < 0:
                pm = prod(conjPs_maps, conjPs_maps, -lam3, (-1.) ** (s + lam3))
            else:
                pm = prod(Ps_maps, Ps_maps, lam3)
            PQ[s + lam3] = self._coll_lm(pm.real) + 1.0j * self._coll_lm(pm.imag)
        if np.imag(beta) == 0:
            return PQ, PQ
        for lam3 in range(-s, s + 1):
            if lam3 < 0:
                pm = prod(Ps_maps, Ps_maps, -lam3, (-1.) ** (s + lam3))
            else:
                pm = prod(conjPs_maps, conjPs_maps, lam3)
            cPQ[s + lam3] = self._coll_lm(pm.real) + 1.0j * self._coll_lm(pm.imag)
        return PQ, cPQ

    def _coll_S_weights(self, s, nu_s):
        return np.asarray([self._calC(s, S, 1.0j * nu_s) * np.exp(1.0j * self._omega_prime(s, 1.0j * nu_s))
                           for S in range(0, 2 * s + 1, 2)], dtype=np.complex128)

    def _convolve_coll_F(self, PQ_vecs, r_weights, s, beta, conjPQ_vecs=None):
        """Sum_S C_S F^beta * [P^beta_{s,lam3} Q] maps for every lam1 (polyspec/tspec_template.py:2192-2283):
        [s+1 (real beta) or 2s+1, N_r, Npix] complex; s = 0 with real beta uses the real part of F."""
        nr = self.N_r
        inds = np.arange(nr, dtype=np.int32)
        nu_s = beta + 1.5
        nF = int(np.max(self.coll_params[beta][:, 1]))
        F = self.d_coll_FLLs[beta]
        nfull = len(self.nLminfilt)
        b = self.base

        def maps(o_re, o_im):
            if bool((o_im != 0.).any()):
                return pixel.r2cstar(b.to_map_vec(o_re.T.contiguous(), lmax=self.nLmax),
                                     b.to_map_vec((1.0j * o_im).T.contiguous(), lmax=self.nLmax))
            return b.to_map_vec(o_re.T.contiguous(), lmax=self.nLmax).to(torch.complex128)

        if s == 0 and np.imag(beta) == 0:
            out = torch.zeros((nfull, nr), dtype=torch.complex128, device=self._dev)
            self.utils.convolve_F_n000_real(PQ_vecs[0], F, r_weights, out, nF, inds)
            out *= (4. * np.pi) ** (3. / 2.)
            return b.to_map_vec(out.T.contiguous(), lmax=self.nLmax).to(torch.complex128)[None]
        Sw = self._coll_S_weights(s, nu_s)
        cPQ = PQ_vecs if conjPQ_vecs is None else conjPQ_vecs
        lams = range(s + 1) if np.imag(beta) == 0 else range(-s, s + 1)
        out = torch.zeros((len(lams), nr, b.Npix), dtype=torch.complex128, device=self._dev)
        for idx, lam1 in enumerate(lams):
            o_re = torch.zeros((nfull, nr), dtype=torch.complex128, device=self._dev)
            o_im = torch.zeros_like(o_re)
            self.utils.convolve_F_general_collider(PQ_vecs, cPQ, F, r_weights, o_re, o_im, s, lam1, nF, Sw, inds)
            if s == 0:
                out[idx] = pixel.r2cstar(b.to_map_vec(o_re.T.contiguous(), lmax=self.nLmax),
                                         b.to_map_vec((1.0j * o_im).T.contiguous(), lmax=self.nLmax))
            else:
                out[idx] = maps(o_re, o_im)
        return out

    def _coll_F_PQ(self, Ps_maps, Q_maps, r_weights, s, beta, conjPs_maps=None):
        """F^beta_L * [P^beta_{s,lam} Q]_LM maps of the (1, 1), (2, 2) and symmetrised (1, 2) pairs
        (polyspec/tspec_template.py:2308-2337): [3, s+1 or 2s+1, N_r, Npix] complex."""
        out = []
        for i1, i2 in ((0, 0), (1, 1), (0, 1)):
            t0 = time.time()
            if np.imag(beta) == 0:
                PQ = self._compute_coll_PQ_vecs(Ps_maps, Q_maps, i1, i2, s, beta, add_sym=(i1 != i2))
                out.append(self._convolve_coll_F(PQ, r_weights, s, beta))
            else:
                PQ, cPQ = self._compute_coll_PQ_vecs(Ps_maps, Q_maps, i1, i2, s, beta, add_sym=(i1 != i2),
                                                     conjPs_maps=conjPs_maps)
                out.append(self._convolve_coll_F(PQ, r_weights, s, beta, conjPQ_vecs=cPQ))
            self._timed('fish_convolve', t0)
        return torch.stack(out)

    def _Q4_contributions_coll(self, Pn1_maps, Q_maps, F_PQ, pq_inds, F_inds, r_weights, weights, n1, beta,
                               conjPn1_maps=None):
        """One Q4 row of a collider template (polyspec/tspec_template.py:2340-2495 with beta_coll): the q_l^X radial
        sum of [P^beta F_PQ]_lm plus the p^beta-weighted sums of the shifted [Q F_PQ]_lm."""
        t0 = time.time()
        b = self.base
        w = np.asarray(r_weights, dtype=np.float64)
        nr = Q_maps.shape[1]
        inds = np.arange(nr, dtype=np.int32)
        out = torch.zeros((1 + 2 * self.pol, len(self.ls)), dtype=torch.complex128, device=self._dev)
        this_nmax = int(np.max(self.coll_params[beta][:, 0]))
        P = self.d_coll_plLXs[beta]
        cplx = np.imag(beta) != 0
        if n1 == 0:
            prod = pixel.compute_productP_all(Pn1_maps[:, 0], F_PQ[:, 0], weights, pq_inds, F_inds)
            lm = b.to_lm_vec(prod, lmax=self.lmax)[:, self.d_lminfilt]
            pixel.integrate_pq(self.d_qlXs, lm.T, self.ls, w, out, inds)
            if cplx:
                prod = pixel.compute_productQ_complex_all(Q_maps, F_PQ, weights, pq_inds, F_inds, 0)
                re = b.to_lm_vec(prod.real.contiguous(), lmax=self.lmax)[:, self.d_lminfilt].T
                im = b.to_lm_vec(prod.imag.contiguous(), lmax=self.lmax)[:, self.d_lminfilt].T
                plus, minus = pixel.complex_to_complex_transpose(re, im)
                pixel.integrate_pq_complex(P[this_nmax], plus, minus, self.ls, w / np.sqrt(4. * np.pi), out, inds)
            else:
                prod = pixel.compute_productQ_real_all(Q_maps, F_PQ, weights, pq_inds, F_inds, 0)
                plus = b.to_lm_vec(prod, lmax=self.lmax)[:, self.d_lminfilt].T
                pixel.integrate_pq(P[this_nmax].real.contiguous(), plus, self.ls, w / np.sqrt(4. * np.pi), out, inds)
            self._timed('fish_deriv', t0)
            return out
        if cplx:
            prod = pixel.compute_productPnmu_all(Pn1_maps, conjPn1_maps, F_PQ, weights, n1, pq_inds, F_inds)
        else:
            prod = pixel.compute_productPnmu_sym_all(Pn1_maps, F_PQ, weights, n1, pq_inds, F_inds)
        lm = b.to_lm_vec(prod, lmax=self.lmax)[:, self.d_lminfilt]
        pixel.integrate_pq(self.d_qlXs, lm.T, self.ls, w, out, inds)
        lmx = min(self.lmax + n1, b.lmax)
        for mu1 in range(-n1, n1 + 1):
            if cplx:
                mu1_index = n1 + mu1
            else:
                if mu1 < 0:
                    continue
                mu1_index = mu1
            if bool((F_PQ[F_inds[0], mu1_index, :, 0].imag != 0).any()):
                prod = pixel.compute_productQ_complex_all(Q_maps, F_PQ, weights, pq_inds, F_inds, mu1_index)
                pm = pixel.complex_to_complex(b.to_lm_vec(prod.real.contiguous(), lmax=lmx),
                                              b.to_lm_vec(prod.imag.contiguous(), lmax=lmx))
                plus, minus = pm[0], pm[1]
            else:
                prod = pixel.compute_productQ_real_all(Q_maps, F_PQ, weights, pq_inds, F_inds, mu1_index)
                plus = b.to_lm_vec(prod, lmax=lmx).T.to(torch.complex128).contiguous()
                minus = plus
            if cplx:
                self.utils.compute_pF_map_complex(plus, minus, P, w, n1, mu1, this_nmax, lmx, out, inds)
            else:
                self.utils.compute_pF_map_real(plus, minus, P.real.contiguous(), w, n1, mu1, this_nmax, lmx, out,
                                               inds)
        self._timed('fish_deriv', t0)
        return out

    def _get_Q4_perms_coll(self, P_maps, Q_maps, F_PQ, r_weights, n1, beta, conjP_maps=None):
        """The four Q4 rows (111, 222, 112, 122) of a collider template (polyspec/tspec_template.py:2521-2554)."""
        rows = (([0], [0], [12.]), ([1], [1], [12.]), ([1, 0], [0, 2], [4., 4.]), ([0, 1], [1, 2], [4., 4.]))
        return torch.stack([self._Q4_contributions_coll(P_maps, Q_maps, F_PQ, p, f, r_weights, w, n1, beta,
                                                        conjP_maps) for p, f, w in rows])

    def _compute_PQ_vecs(self, Pn3_maps, Q_maps, i, j, n3=0, add_sym=False):
        """[P Q]_LM(r) of polyspec/tspec_template.py:1967-2010 for n3 = 0, [N_r, nlm(nLmax)]."""
        assert n3 == 0
        if add_sym:
            prod = pixel.multiplyRR_sym(Q_maps[j], Pn3_maps[i, 0], Q_maps[i], Pn3_maps[j, 0])
        else:
            prod = pixel.multiplyRR(Q_maps[j], Pn3_maps[i, 0])
        return self.base.to_lm_vec(prod, lmax=self.nLmax)

    def _F_PQ(self, Pn3_maps, Q_maps, r_weights):
        """F_L * [P Q]_LM maps for the (1, 1), (2, 2) and symmetrised (1, 2) pairs
        (polyspec/tspec_template.py:2287-2306 and :2142-2163, n1 = n3 = n = 0): [3, N_r, Npix] real."""
        out = []
        for i1, i2 in ((0, 0), (1, 1), (0, 1)):
            t0 = time.time()
            PQ = self._compute_PQ_vecs(Pn3_maps, Q_maps, i1, i2, 0, add_sym=(i1 != i2))
            conv = self._tau_convolve(PQ, r_weights)
            out.append(self.base.to_map_vec(conv, lmax=self.nLmax))
            self._timed('fish_convolve', t0)
        return torch.stack(out)

    def _Q4_contributions(self, P_maps, Q_maps, F_PQ, pq_inds, F_inds, r_weights, weights):
        """One Q4 row of the local tauNL derivative (polyspec/tspec_template.py:2341-2405, n1 = 0):
        q_l^X-weighted radial sum of [P F_PQ]_lm plus p_l^X-weighted radial sum of [Q F_PQ]_lm."""
        t0 = time.time()
        w = np.asarray(r_weights, dtype=np.float64)
        prod = pixel.compute_product_real_all(P_maps[:, 0], F_PQ, weights, pq_inds, F_inds)
        lm = self.base.to_lm_vec(prod, lmax=self.lmax)[:, self.d_lminfilt].contiguous()
        out = self.utils.radial_sum(lm, 0.5 * w, self.d_qlXs)
        prod = pixel.compute_product_real_all(Q_maps, F_PQ, weights, pq_inds, F_inds)
        lm = self.base.to_lm_vec(prod, lmax=self.lmax)[:, self.d_lminfilt].contiguous()
        out = out + self.utils.radial_sum(lm, 0.5 * (w / np.sqrt(4. * np.pi)), self.d_plLXs[self.nmax])
        self._timed('fish_deriv', t0)
        return out

    def _get_Q4_perms(self, P_maps, Q_maps, F_PQ, r_weights):
        """The four Q4 rows (111, 222, 112, 122) of polyspec/tspec_template.py:2521-2554."""
        rows = (([0], [0], [12.]), ([1], [1], [12.]), ([1, 0], [0, 2], [4., 4.]), ([0, 1], [1, 2], [4., 4.]))
        return torch.stack([self._Q4_contributions(P_maps, Q_maps, F_PQ, p, f, r_weights, w) for p, f, w in rows])

    def _compute_PQ_vecs_n(self, Pn3_maps, Q_maps, i, j, n3, add_sym=False):
        """[P_{n3,mu3} Q]_LM for mu3 = -n3..n3 (polyspec/tspec_template.py:1967-2010, n3 > 0), in the
        reference's layout [2 n3 + 1, len(Ls), N_r]."""
        nl = int(np.sum(self.nLminfilt))
        sel = self.d_nLminfilt_idx
        if n3 == 0:
            if add_sym:
                prod = pixel.multiplyRR_sym(Q_maps[j], Pn3_maps[i, 0], Q_maps[i], Pn3_maps[j, 0])
            else:
                prod = pixel.multiplyRR(Q_maps[j], Pn3_maps[i, 0])
            return self.base.to_lm_vec(prod, lmax=self.nLmax)[:, sel].T[None].contiguous()
        PQ = torch.zeros((2 * n3 + 1, nl, Q_maps.shape[1]), dtype=torch.complex128, device=self._dev)
        for mu3 in range(n3 + 1):
            if add_sym:
                prod = pixel.multiplyRC_sym(Q_maps[j], Pn3_maps[i, mu3], Q_maps[i], Pn3_maps[j, mu3])
            else:
                prod = pixel.multiplyRC(Q_maps[j], Pn3_maps[i, mu3])
            lm = lambda x: self.base.to_lm_vec(x.contiguous(), lmax=self.nLmax)[:, sel].T
            if mu3 == 0 and n3 % 2 == 0:
                PQ[n3] = lm(prod.real)
            elif mu3 == 0:
                PQ[n3] = 1.0j * lm(prod.imag)
            else:
                pr, pi = lm(prod.real), 1.0j * lm(prod.imag)
                PQ[n3 + mu3] = pr + pi
                PQ[n3 - mu3] = (-1.) ** (n3 - mu3) * (pr - pi)
        return PQ

    def _convolve_F_n(self, PQ, r_weights, n1, n3=None, n=0):
        """F convolution of the [P_{n3} Q] vectors (polyspec/tspec_template.py:2142-2190): convolve_F_n0 for n = 0
        (n1 = n3), convolve_F_general otherwise; [n1 + 1, N_r, Npix] complex maps, mu1 = 0..n1."""
        n3 = n1 if n3 is None else n3
        nr = PQ.shape[2]
        inds = np.arange(nr, dtype=np.int32)
        out = torch.zeros((n1 + 1, nr, self.base.Npix), dtype=torch.complex128, device=self._dev)
        nfull = len(self.nLminfilt)
        for mu1 in range(n1 + 1):
            o_re = torch.zeros((nfull, nr), dtype=torch.complex128, device=self._dev)
            o_im = torch.zeros_like(o_re)
            if n == 0:
                self.utils.convolve_F_n0(PQ[n1 - mu1], PQ[n1 + mu1], self.d_FLLs, r_weights, o_re, o_im, n1, mu1,
                                         self.nmax_F, inds)
            else:
                self.utils.convolve_F_general(PQ, self.d_FLLs, r_weights, o_re, o_im, n1, n3, n, mu1, inds)
            if bool((o_im != 0.).any()):
                out[mu1] = pixel.r2cstar(self.base.to_map_vec(o_re.T.contiguous(), lmax=self.nLmax),
                                         self.base.to_map_vec((1.0j * o_im).T.contiguous(), lmax=self.nLmax))
            else:
                out[mu1] = self.base.to_map_vec(o_re.T.contiguous(), lmax=self.nLmax)
        return out

    def _F_PQ_n(self, Pn3_maps, Q_maps, r_weights, n1, n3=None, n=0):
        """F * [P_{n3,mu} Q] maps of the (1, 1), (2, 2) and symmetrised (1, 2) pairs for (n1, n3, n) other than
        (0, 0, 0) (polyspec/tspec_template.py:2287-2306): [3, n1 + 1, N_r, Npix] complex."""
        n3 = n1 if n3 is None else n3
        out = []
        for i1, i2 in ((0, 0), (1, 1), (0, 1)):
            t0 = time.time()
            PQ = self._compute_PQ_vecs_n(Pn3_maps, Q_maps, i1, i2, n3, add_sym=(i1 != i2))
            out.append(self._convolve_F_n(PQ, r_weights, n1, n3, n))
            self._timed('fish_convolve', t0)
        return torch.stack(out)

    def _Q4_contributions_n(self, Pn1_maps, Q_maps, F_PQ, pq_inds, F_inds, r_weights, weights, n1):
        """One Q4 row for n1 > 0 (polyspec/tspec_template.py:2405-2505): the q_l^X radial sum of
        [Sum_mu P_{n1,mu} F_PQ]_lm plus, per mu1, the Gaunt-weighted p_lL^X sums of the shifted [Q F_PQ]_lm."""
        t0 = time.time()
        b = self.base
        w = np.asarray(r_weights, dtype=np.float64)
        nr = Q_maps.shape[1]
        inds = np.arange(nr, dtype=np.int32)
        out = torch.zeros((1 + 2 * self.pol, len(self.ls)), dtype=torch.complex128, device=self._dev)
        prod = pixel.compute_productPnmu_sym_all(Pn1_maps, F_PQ, weights, n1, pq_inds, F_inds)
        P_FPQ = b.to_lm_vec(prod, lmax=self.lmax)[:, self.d_lminfilt]
        pixel.integrate_pq(self.d_qlXs, P_FPQ.T, self.ls, w, out, inds)
        lmx = min(self.lmax + n1, b.lmax)
        for mu1 in range(n1 + 1):
            if bool((F_PQ[F_inds[0], mu1, :, 0].imag != 0).any()):
                prod = pixel.compute_productQ_complex_all(Q_maps, F_PQ, weights, pq_inds, F_inds, mu1)
                pm = pixel.complex_to_complex(b.to_lm_vec(prod.real.contiguous(), lmax=lmx),
                                              b.to_lm_vec(prod.imag.contiguous(), lmax=lmx))
                plus, minus = pm[0], pm[1]
            else:
                prod = pixel.compute_productQ_real_all(Q_maps, F_PQ, weights, pq_inds, F_inds, mu1)
                plus = b.to_lm_vec(prod, lmax=lmx).T.contiguous()
                minus = plus
            self.utils.compute_pF_map_real(plus, minus, self.d_plLXs, w, n1, mu1, self.nmax, lmx, out, inds)
        self._timed('fish_deriv', t0)
        return out

    def _get_Q4_perms_n(self, P_maps, Q_maps, F_PQ, r_weights, n1):
        """The four Q4 rows (111, 222, 112, 122) for n1 > 0 (polyspec/tspec_template.py:2521-2554)."""
        rows = (([0], [0], [12.]), ([1], [1], [12.]), ([1, 0], [0, 2], [4., 4.]), ([0, 1], [1, 2], [4., 4.]))
        return torch.stack([self._Q4_contributions_n(P_maps, Q_maps, F_PQ, p, f, r_weights, w, n1)
                            for p, f, w in rows])

    # ------------------------------------------------------------------ numerator
    def Tl_numerator(self, data, include_disconnected_term=True, verb=False, input_type='map'):
        """Numerator of the unwindowed trispectrum estimator (polyspec/tspec_template.py:1338-1955)."""
        t_start = time.time()
        self._check_sampling()
        if not hasattr(self, 'preload') and include_disconnected_term:
            raise Exception("Need to generate or specify bias simulations!")
        if self.pol:
            assert len(data) == 3, "Data must contain T, Q, U components!"
        else:
            assert (len(data) == 1 and len(data[0]) == self.base.Npix) or len(data) == self.base.Npix, \
                "Data must contain T only!"
        if hasattr(self, 't0_num') and include_disconnected_term:
            compute_t0 = False
            if verb:
                print("Using precomputed t0 term")
        else:
            compute_t0 = True
        t0 = time.time()
        d = self.base._in(data, torch.float64 if input_type == 'map' else torch.complex128)[0]
        h_data_lm = self._sinv_filt(d, input_type)
        self._timed('Sinv', t0)
        proc_maps = self._apply_all_filters(h_data_lm)
        A_pix = self.base.A_pix
        t4_num = np.zeros(len(self.templates))
        if not include_disconnected_term:
            print("## No subtraction of (parity-conserving) disconnected terms performed!")
        else:
            t2_num = np.zeros(len(self.templates))
            if compute_t0:
                t0_num = np.zeros(len(self.templates))
        if verb:
            print("# Assembling trispectrum numerator (4-field term)")
        Phi_dd = None
        A_dd = {}
        for ii, t in enumerate(self.templates):
            if t == 'gNL-loc':
                t0 = time.time()
                t4_num[ii] = 9. / 100. * self.utils.gnl_loc_sum(self.r_weights[t], proc_maps['p00'], proc_maps['q']) \
                    * 4. * A_pix * (4. * np.pi) ** 1.5
                self._timed('gNL_summation', t0)
            if t == 'tauNL-loc':
                if 0 not in A_dd:
                    A_dd[0] = self._A_maps(proc_maps, proc_maps, 0)
                t4_num[ii] = 1. / 24. * self._tau_sum(A_dd, A_dd, self.r_weights[t], 0, 0, 0) * 12. \
                    * (4. * np.pi) ** (3. / 2.)
            if _is_direc(t):
                tau = 0.
                for n1, n3, n, wt in self._direc_parts(t):
                    for nn in (n1, n3):
                        if nn not in A_dd:
                            A_dd[nn] = self._A_maps(proc_maps, proc_maps, nn)
                    tau += wt * self._tau_sum(A_dd, A_dd, self.r_weights[t], n1, n3, n)
                t4_num[ii] = tau / 48. * 24.
            if _is_coll(t):
                # collider tauNL (polyspec/tspec_template.py:1489-1518): [P^beta Q] maps of beta and, for a
                # heavy particle, of its conjugate; the sum takes the real part
                s_, x = _coll_parse(t)
                betas = [-1.5 + x] if 'tauNL-light' in t else [-1.5 - 1.0j * x, -1.5 + 1.0j * x]
                for beta in betas:
                    if _ckey_s(s_, beta) not in A_dd:
                        A_dd[_ckey_s(s_, beta)] = self._A_maps(proc_maps, proc_maps, s_, beta=beta)
                t4_num[ii] = self._tau_sum_collider(A_dd, A_dd, self.r_weights[t], s_, betas[0]) / 24. * 12.
            if t in ('gNL-con', 'gNL-dotdot', 'gNL-dotdel', 'gNL-deldel'):
                t0 = time.time()
                t4_num[ii] = self._gnl_shape_sum(t, proc_maps) * A_pix
                self._timed('gNL_summation', t0)
            if t == 'lensing':
                Phi_dd = self._compute_lensing_Phi(proc_maps, proc_maps)
                w = self._lens_Ls()
                t0 = time.time()
                t4_num[ii] = 1. / 24. * float(torch.sum(w * (Phi_dd * Phi_dd.conj()).real)) * 12.
                self._timed('lensing_summation', t0)
            if t == 'point-source':
                t0 = time.time()
                t4_num[ii] = 1. / 24. * float(torch.sum(proc_maps['u'][0].real ** 4.)) * A_pix
                self._timed('gNL_summation', t0)

        if include_disconnected_term:
            for isim in range(self.N_it):
                if verb:
                    print("# Assembling 2-field%s trispectrum numerator for simulation pair %d of %d"
                          % ("" if not compute_t0 else " and 0-field", isim + 1, self.N_it))
                if self.preload:
                    pa, pb = self.proc_a_maps[isim], self.proc_b_maps[isim]
                else:
                    pa, pb = self.load_sim_data(isim)
                A_aa, A_bb, A_ad, A_bd, A_ab = {}, {}, {}, {}, {}
                for ii, t in enumerate(self.templates):
                    if _is_direc(t):
                        w = self.r_weights[t]
                        t2, t0s = 0., 0.
                        for n1, n3, n, wt in self._direc_parts(t):
                            tmp = 0.
                            for A_xx, A_xd, px in ((A_aa, A_ad, pa), (A_bb, A_bd, pb)):
                                for nn in np.unique([n1, n3]):
                                    if nn not in A_xx:
                                        A_xx[nn] = self._A_maps(px, px, nn)
                                        A_xd[nn] = self._A_maps(px, proc_maps, nn, add_sym=True)
                                if n1 == n3:
                                    tmp += 2 * self._tau_sum(A_xx, A_dd, w, n1, n3, n)
                                else:
                                    tmp += self._tau_sum(A_xx, A_dd, w, n1, n3, n) \
                                        + self._tau_sum(A_dd, A_xx, w, n1, n3, n)
                                tmp += self._tau_sum(A_xd, A_xd, w, n1, n3, n)
                            t2 += wt * tmp
                            if compute_t0:
                                tmp = 0.
                                for nn in np.unique([n1, n3]):
                                    if nn not in A_ab:
                                        A_ab[nn] = self._A_maps(pa, pb, nn, add_sym=True)
                                if n1 == n3:
                                    tmp += 2 * self._tau_sum(A_aa, A_bb, w, n1, n3, n)
                                else:
                                    tmp += self._tau_sum(A_aa, A_bb, w, n1, n3, n) \
                                        + self._tau_sum(A_bb, A_aa, w, n1, n3, n)
                                tmp += self._tau_sum(A_ab, A_ab, w, n1, n3, n)
                                t0s += wt * tmp
                        t2_num[ii] += -1. / 48. * t2 * 6. / self.N_it / 2. * 4.
                        if compute_t0:
                            t0_num[ii] += 1. / 48. * t0s * 3 / self.N_it * 4.
                    if _is_coll(t):
                        # collider 2- and 0-field terms (polyspec/tspec_template.py:1817-1894)
                        s_, x = _coll_parse(t)
                        w = self.r_weights[t]
                        betas = [-1.5 + x] if 'tauNL-light' in t else [-1.5 - 1.0j * x, -1.5 + 1.0j * x]
                        tau = 0.
                        for A_xx, A_xd, px in ((A_aa, A_ad, pa), (A_bb, A_bd, pb)):
                            for beta in betas:
                                if _ckey_s(s_, beta) not in A_xx:
                                    A_xx[_ckey_s(s_, beta)] = self._A_maps(px, px, s_, beta=beta)
                                    A_xd[_ckey_s(s_, beta)] = self._A_maps(px, proc_maps, s_, add_sym=True,
                                                                           beta=beta)
                            tau += 2 * self._tau_sum_collider(A_xx, A_dd, w, s_, betas[0])
                            tau += self._tau_sum_collider(A_xd, A_xd, w, s_, betas[0])
                        t2_num[ii] += -1. / 24. * tau * 6. / self.N_it / 2. * 2.
                        if compute_t0:
                            for beta in betas:
                                if _ckey_s(s_, beta) not in A_ab:
                                    A_ab[_ckey_s(s_, beta)] = self._A_maps(pa, pb, s_, add_sym=True, beta=beta)
                            tau = 2 * self._tau_sum_collider(A_aa, A_bb, w, s_, betas[0])
                            tau += self._tau_sum_collider(A_ab, A_ab, w, s_, betas[0])
                            t0_num[ii] += 1. / 24. * tau * 3 / self.N_it * 2.
                    if t == 'tauNL-loc':
                        w = self.r_weights[t]
                        if 0 not in A_aa:
                            A_aa[0] = self._A_maps(pa, pa, 0)
                            A_ad[0] = self._A_maps(pa, proc_maps, 0, add_sym=True)
                        tau = 4 * self._tau_sum(A_aa, A_dd, w, 0, 0, 0)
                        tau += 2 * self._tau_sum(A_ad, A_ad, w, 0, 0, 0)
                        if 0 not in A_bb:
                            A_bb[0] = self._A_maps(pb, pb, 0)
                            A_bd[0] = self._A_maps(pb, proc_maps, 0, add_sym=True)
                        tau += 4 * self._tau_sum(A_bb, A_dd, w, 0, 0, 0)
                        tau += 2 * self._tau_sum(A_bd, A_bd, w, 0, 0, 0)
                        t2_num[ii] += -1. / 24. * tau * 6 / self.N_it / 2. * (4. * np.pi) ** (3. / 2.)
                        if compute_t0:
                            if 0 not in A_ab:
                                A_ab[0] = self._A_maps(pa, pb, 0, add_sym=True)
                            tau = 4 * self._tau_sum(A_aa, A_bb, w, 0, 0, 0)
                            tau += 2 * self._tau_sum(A_ab, A_ab, w, 0, 0, 0)
                            t0_num[ii] += 1. / 24. * tau * 3 / self.N_it * (4. * np.pi) ** (3. / 2.)
                    if t == 'gNL-loc':
                        t0 = time.time()
                        w = self.r_weights[t]
                        perm = lambda m12, m34: self.utils.gnl_loc_disc_sum(w, m12['p00'], m34['p00'], m12['q'],
                                                                            m34['q'])
                        summ = perm(proc_maps, pa) + perm(proc_maps, pb)
                        t2_num[ii] += -54. / 100. * summ / self.N_it * A_pix * (4. * np.pi) ** 1.5
                        if compute_t0:
                            t0_num[ii] += 54. / 100. * perm(pa, pb) / self.N_it * A_pix * (4. * np.pi) ** 1.5
                        self._timed('gNL_summation', t0)
                    if t in ('gNL-con', 'gNL-dotdot', 'gNL-dotdel', 'gNL-deldel'):
                        t0 = time.time()
                        t2_num[ii] += -self._gnl_shape_disc(t, proc_maps, pa, pb) / self.N_it * A_pix
                        if compute_t0:
                            t0_num[ii] += self._gnl_shape_disc(t, pb, pa) / self.N_it * A_pix
                        self._timed('gNL_summation', t0)
                    if t == 'lensing':
                        w = self._lens_Ls()
                        Phi_aa = self._compute_lensing_Phi(pa, pa)
                        Phi_ad = self._compute_lensing_Phi(pa, proc_maps, add_sym=True)
                        Phi_sum = 4. * Phi_aa * Phi_dd.conj() + 2. * Phi_ad * Phi_ad.conj()
                        Phi_bb = self._compute_lensing_Phi(pb, pb)
                        Phi_bd = self._compute_lensing_Phi(pb, proc_maps, add_sym=True)
                        Phi_sum += 4. * Phi_bb * Phi_dd.conj() + 2. * Phi_bd * Phi_bd.conj()
                        t0 = time.time()
                        t2_num[ii] += -1. / 24. * float(torch.sum(w * Phi_sum).real) * 3. / self.N_it
                        self._timed('lensing_summation', t0)
                        if compute_t0:
                            Phi_ab = self._compute_lensing_Phi(pa, pb, add_sym=True)
                            Phi_sum = 4. * Phi_aa * Phi_bb.conj() + 2. * Phi_ab * Phi_ab.conj()
                            t0 = time.time()
                            t0_num[ii] += 1. / 24. * float(torch.sum(w * Phi_sum).real) * 3. / self.N_it
                            self._timed('lensing_summation', t0)
                    if t == 'point-source':
                        t0 = time.time()
                        perm = lambda m12, m34: float(torch.sum(m12['u'][0].real ** 2. * m34['u'][0].real ** 2.))
                        summ = perm(proc_maps, pa) + perm(proc_maps, pb)
                        t2_num[ii] += -3. / 24. * summ / self.N_it * A_pix
                        if compute_t0:
                            t0_num[ii] += 3. / 24. * perm(pa, pb) / self.N_it * A_pix
                        self._timed('gNL_summation', t0)
            if not compute_t0:
                t0_num = self.t0_num
            else:
                self.t0_num = t0_num
        self.timers['numerator'] += time.time() - t_start
        if include_disconnected_term:
            return t4_num + t2_num + t0_num
        return t4_num

    def _gnl_shape_sum(self, t, m):
        """4-field sums of gNL-con and the EFTI shapes without A_pix (polyspec/tspec_template.py:1394-1420)."""
        u = self.utils
        if t == 'gNL-con':
            return 9. / 25. * u.gnl_con_sum(self.r_weights[t], m['r'])
        w, tau = self.rtau_weights[t], self.rtau_arr[:, 1]
        if t == 'gNL-dotdot':
            return 384. / 25. * u.gnl_dotdot_sum(w, tau, m['a'])
        if t == 'gNL-dotdel':
            return 288. / 325. * u.gnl_dotdel_sum(w, tau, m['a'], m['b'], m['c']) * 12
        return 1728. / 2575. * u.gnl_deldel_sum(w, m['b'], m['c']) * 6

    def _gnl_shape_disc(self, t, d, a, b=None):
        """Disconnected sums of gNL-con and the EFTI shapes without A_pix (polyspec/tspec_template.py:1582-1660):
        with b, the 2-field sum over the pairs (d, a) and (d, b) (to be subtracted); without, the
        0-field sum of the pair (d, a), called with d the second simulation and a the first."""
        u = self.utils
        pairs = [(d, a), (d, b)] if b is not None else [(d, a)]
        summ = 0.
        if t == 'gNL-con':
            w = self.r_weights[t]
            for x, y in pairs:
                summ += u.gnl_con_disc_sum(w, x['r'], y['r'])
            return 27. / 25. * summ
        w, tau = self.rtau_weights[t], self.rtau_arr[:, 1]
        if t == 'gNL-dotdot':
            for x, y in pairs:
                summ += u.gnl_dotdot_disc_sum(w, tau, x['a'], y['a'])
            return 1152. / 25. * summ
        if t == 'gNL-dotdel':
            def perm(m1, m2, m3, m4):
                return u.gnl_dotdel_disc_sum(w, tau, m1['a'], m2['a'], m3['b'], m4['b'], m3['c'], m4['c'])
            for x, y in pairs:  # x is the data (or the first simulation), y the simulation
                summ += 2 * perm(y, y, x, x) + 8 * perm(y, x, y, x) + 2 * perm(x, x, y, y)
            return 864. / 325. * summ

        def perm(m1, m2, m3, m4):
            return u.gnl_deldel_disc_sum(w, m1['b'], m2['b'], m3['b'], m4['b'], m1['c'], m2['c'], m3['c'], m4['c'])
        for x, y in pairs:
            summ += 2 * perm(y, y, x, x) + 4 * perm(y, x, y, x)
        return 5184. / 2575. * summ

    # ------------------------------------------------------------------ Fisher matrix
    def _transform_maps(self, map123, flXs, weights, spin=0):
        """Sum_i w_i M_LM f^X_L(i) for maps M [N, Npix] (polyspec/tspec_template.py:2575-2588): real maps
        through a spin-0 adjoint; complex (+1) maps through the spin-1 adjoint of (M, conj M),
        averaging the +1 and -1 harmonics."""
        t0 = time.time()
        if spin == 0:
            lm_map = self.base.to_lm_vec(map123, lmax=self.lmax)[:, self.d_lminfilt].contiguous()
            out = self.utils.radial_sum(lm_map, weights, flXs)
        elif spin == 1:
            lm_map = self.base.to_lm_vec(torch.stack([map123, map123.conj()]), spin=1, lmax=self.lmax)
            out = self.utils.radial_sum_spin1(lm_map[:, :, self.d_lminfilt].contiguous(), weights, flXs)
        else:
            raise Exception(f"Wrong spin s = {spin}!")
        self._timed('fish_deriv', t0)
        return out

    def _tau_pow(self, n):
        """tau_i^n over the (r, tau) samples, shaped to scale an [l, X, i] integral array."""
        return torch.as_tensor(self.rtau_arr[:, 1], device=self._dev)[None, None, :] ** n

    def _dotdel_Q(self, A, B, C, w):
        """Q-derivative rows (111, 222, 112, 122) of gNL-dotdel (polyspec/tspec_template.py:2768-2801)."""
        u, tm = self.utils, self._transform_maps
        t2 = self._tau_pow(2.)
        fa, fb, fc = self.d_alXs * t2, self.d_blXs * t2, self.d_clXs * t2
        Q = torch.zeros((4, 1 + 2 * self.pol, len(self.ls)), dtype=torch.complex128, device=self._dev)
        for k, i in ((0, 0), (1, 1)):
            Q[k] = 41472. / 325. * tm(u.multiplyCC(A[i], B[i], C[i]), fa, w)
            Q[k] += 41472. / 325. * tm(u.multiply(A[i], A[i], B[i]), fb, w)
            Q[k] += 41472. / 325. * tm(u.multiplyC(A[i], A[i], C[i]), fc, w, spin=1)
        for k, (i, j) in ((2, (0, 1)), (3, (1, 0))):
            Q[k] = 13824. / 325. * tm(u.multiplyCC_asym(A[i], A[j], B[i], B[j], C[i], C[j]), fa, w)
            Q[k] += 13824. / 325. * tm(u.multiply_asym(A[i], A[j], B[i], B[j]), fb, w)
            Q[k] += 13824. / 325. * tm(u.multiplyC_asym(A[i], A[j], C[i], C[j]), fc, w, spin=1)
        return Q

    def _deldel_Q(self, B, C, w):
        """Q-derivative rows (111, 222, 112, 122) of gNL-deldel (polyspec/tspec_template.py:2803-2841)."""
        u, tm = self.utils, self._transform_maps
        fb, fc = self.d_blXs, self.d_clXs
        quad = {(0, 0): u.multiply2(B[0], B[0], C[0], C[0]), (0, 1): u.multiply2(B[0], B[1], C[0], C[1]),
                (1, 1): u.multiply2(B[1], B[1], C[1], C[1])}
        Q = torch.zeros((4, 1 + 2 * self.pol, len(self.ls)), dtype=torch.complex128, device=self._dev)

        def term(coef, i, q):
            return coef * tm(u.multiply2R(B[i], q), fb, w) + coef * tm(u.multiply2C(C[i], q), fc, w, spin=1)
        Q[0] = term(248772. / 2575., 0, quad[0, 0])
        Q[1] = term(248772. / 2575., 1, quad[1, 1])
        Q[2] = term(82944. / 2575., 1, quad[0, 0]) + term(165888. / 2575., 0, quad[0, 1])
        Q[3] = term(82944. / 2575., 0, quad[1, 1]) + term(165888. / 2575., 1, quad[0, 1])
        return Q

    def _weight_Q_maps(self, tmp_Q, weighting='Ainv'):
        """S^-1 P weighting (A^-1 branch) or m weights (S^-1 branch) of Q rows
        [R, 1+2 pol, nlm_filt] (polyspec/tspec_template.py:2556-2572), batched."""
        if weighting == 'Sinv':
            return tmp_Q * self.d_m_weight
        t0 = time.time()
        full = self._full_lm(self.d_beam_lm * tmp_Q, self.lmax)
        R = len(full)
        if self.ones_mask:
            out = torch.stack([self.applySinv(full[r], input_type='harmonic', lmax=self.lmax) for r in range(R)])
        else:
            maps = torch.stack([self.base.to_map(full[r], lmax=self.lmax) for r in range(R)]) \
                if full.shape[1] not in (1, 3) else self.base.to_map_batch(full, lmax=self.lmax)
            maps = maps * self.d_mask[None]
            if hasattr(self.applySinv, 'batched'):
                out = self.applySinv.batched(maps, lmax=self.lmax)
            else:
                out = torch.stack([self.applySinv(m, lmax=self.lmax) for m in maps])
        self._timed('Sinv', t0)
        return out[:, :, self.d_lminfilt]

    def _lensing_Q(self, U_maps, V_maps):
        """Lensing Q derivatives [4, 1+2 pol, nlm_filt] (polyspec/tspec_template.py:2908-3014)."""
        b = self.base
        fields1 = {'u': U_maps[0], 'v': V_maps[0]}
        fields2 = {'u': U_maps[1], 'v': V_maps[1]}
        Ls = self.base.l_arr[(self.base.l_arr >= self.Lmin_lens) * (self.base.l_arr <= self.Lmax_lens)]
        wL = torch.as_tensor(Ls * (Ls + 1.) * np.asarray(self.C_phi)[Ls], device=self._dev)
        nL = (self.Lmax_lens + 1) * (self.Lmax_lens + 2) // 2

        def W(m1, m2, add_sym=False):
            tmp = torch.zeros(nL, dtype=torch.complex128, device=self._dev)
            tmp[self.d_Lminfilt_lens] = wL * self._compute_lensing_Phi(m1, m2, add_sym=add_sym)
            return b.to_map_spin(tmp, -tmp, spin=1, lmax=self.Lmax_lens)[0]

        W_11 = W(fields1, fields1)
        W_12sym = W(fields1, fields2, add_sym=True)
        W_22 = W(fields2, fields2)
        ls = torch.as_tensor(self.ls.astype(np.float64), device=self._dev)
        lsi = torch.as_tensor(self.ls, device=self._dev)
        Cl = {k: torch.as_tensor(np.asarray(v, dtype=np.float64), device=self._dev)[lsi]
              for k, v in self.C_lens_weight.items()}
        lpref0 = 0.5 * torch.sqrt(ls * (ls + 1.))
        if self.pol:
            lprefp1 = 0.25 * torch.sqrt((ls + 2.) * (ls - 1.))
            lprefm1 = 0.25 * torch.sqrt((ls - 2.) * (ls + 3.))
        f = self.d_lminfilt

        def spin_lm(m, s):
            pm = b.to_lm_spin(m, m.conj(), spin=s, lmax=self.lmax)
            return pm[0][f], pm[1][f]

        def get_Q(fields, Wm):
            Q = torch.zeros((1 + 2 * self.pol, len(self.ls)), dtype=torch.complex128, device=self._dev)
            m = torch.real(fields['v'][0] * Wm)
            Q[0] = -b.to_lm(m[None], lmax=self.lmax)[0][f]
            if self.pol:
                m = fields['v'][1] * Wm - fields['v'][2] * Wm.conj()
                p, mi = spin_lm(m, 2)
                Q[1] = -0.25 * (p + mi)
                Q[2] = 0.25j * (p - mi)
            m = fields['u'][0] * Wm
            p, mi = spin_lm(m, 1)
            tp = p - mi
            Q[0] += lpref0 * Cl['TT'] * tp
            if self.pol:
                Q[1] += lpref0 * Cl['TE'] * tp
                for X, sgn_i in ((1, False), (2, True)):
                    for s, lpref, conj in ((1, lprefp1, True), (3, lprefm1, False)):
                        m = -fields['u'][X] * Wm.conj() if conj else fields['u'][X] * Wm
                        p, mi = spin_lm(m, s)
                        if not sgn_i:   # Z = E
                            base_ = lpref * (p - mi)
                            Q[0] += Cl['TE'] * base_
                            Q[1] += Cl['EE'] * base_
                            Q[2] += lpref * (-1.0j) * Cl['BB'] * (p + mi)
                        else:           # Z = B
                            base_ = lpref * 1.0j * (p + mi)
                            Q[0] += Cl['TE'] * base_
                            Q[1] += Cl['EE'] * base_
                            Q[2] += lpref * Cl['BB'] * (p - mi)
            return Q / 2.

        out = torch.zeros((4, 1 + 2 * self.pol, len(self.ls)), dtype=torch.complex128, device=self._dev)
        out[0] += 12 * get_Q(fields1, W_11)
        out[1] += 12 * get_Q(fields2, W_22)
        out[2] += 4 * get_Q(fields1, W_12sym)
        out[2] += 4 * get_Q(fields2, W_11)
        out[3] += 4 * get_Q(fields2, W_12sym)
        out[3] += 4 * get_Q(fields1, W_22)
        return out

    def compute_fisher_contribution(self, seed, verb=False, a_lms=None):
        """Fisher contribution of one pair of GRFs (polyspec/tspec_template.py:2590-3052).

        ``a_lms`` (two beam-deconvolved harmonic fields) may replace the fields drawn
        from ``seed``."""
        t_start = time.time()
        self._check_sampling()
        print("Computing Fisher matrix with seed %d" % seed)
        b = self.base
        nt = len(self.templates)
        t0 = time.time()
        if a_lms is None:
            a_lms = []
            for ii in range(2):
                if self.ones_mask:
                    a_lms.append(b.generate_data(seed=seed + int((1 + ii) * 1e9), output_type='harmonic',
                                                 lmax=self.lmax, deconvolve_beam=True))
                else:
                    a_lms.append(b.generate_data(seed=seed + int((1 + ii) * 1e9), output_type='harmonic',
                                                 deconvolve_beam=True))
        a_lms = [b._in(a, torch.complex128)[0] for a in a_lms]
        self._timed('fish_grfs', t0)

        def compute_Q4(weighting):
            t0 = time.time()
            if weighting == 'Sinv':
                if self.ones_mask:
                    beam = b.dev('beam_lm', self.lmax)
                    U = [self._sinv_filt(beam * a, 'harmonic') for a in a_lms]
                else:
                    U = [self._sinv_filt(self.d_mask * b.to_map(b.dev('beam_lm') * a)) for a in a_lms]
                self._timed('Sinv', t0)
            else:
                if self.ones_mask:
                    U = [b.applyAinv(a, input_type='harmonic', lmax=self.lmax)[:, self.d_lminfilt].contiguous()
                         for a in a_lms]
                else:
                    U = [b.applyAinv(a, input_type='harmonic')[:, self.d_lfilt].contiguous() for a in a_lms]
                self._timed('Ainv', t0)
            if 'q' in self.to_compute:
                Q_maps = self._filter_pair(U, 'Q')
            if 'r' in self.to_compute:
                R_maps = self._filter_pair(U, 'R')
            if 'a' in self.to_compute:
                A_maps = self._filter_pair(U, 'A')
            if 'b' in self.to_compute:
                B_maps = self._filter_pair(U, 'B')
            if 'c' in self.to_compute:
                C_maps = self._filter_pair(U, 'C')
            if 'u' in self.to_compute:
                U_maps = self._filter_pair(U, 'U')
            if 'v' in self.to_compute:
                V_maps = self._filter_pair(U, 'V')
            if len(self.p_inds) > 0:
                P_maps = self._filter_pair(U, 'P')
            if len(self.coll_params) > 0:
                coll_P = self._filter_pair(U, 'coll-P')
            Qs = torch.zeros((4, nt, 1 + 2 * self.pol, len(self.ls)), dtype=torch.complex128, device=self._dev)
            for ii, t in enumerate(self.templates):
                if t == 'gNL-loc':
                    w = self.r_weights[t]
                    P0 = P_maps[0][:, 0] * np.sqrt(4. * np.pi)
                    p = self.d_plLXs[self.nmax]
                    q = self.d_qlXs
                    u = self.utils
                    Qs[0, ii] = 162. / 25. * self._transform_maps(u.multiply(P0[0], P0[0], Q_maps[0]), p, w)
                    Qs[0, ii] += 54. / 25. * self._transform_maps(u.multiply(P0[0], P0[0], P0[0]), q, w)
                    Qs[1, ii] = 162. / 25. * self._transform_maps(u.multiply(P0[1], P0[1], Q_maps[1]), p, w)
                    Qs[1, ii] += 54. / 25. * self._transform_maps(u.multiply(P0[1], P0[1], P0[1]), q, w)
                    Qs[2, ii] = 54. / 25. * self._transform_maps(u.multiply_asym(P0[0], P0[1], Q_maps[0], Q_maps[1]),
                                                                 p, w)
                    Qs[2, ii] += 54. / 25. * self._transform_maps(u.multiply(P0[0], P0[0], P0[1]), q, w)
                    Qs[3, ii] = 54. / 25. * self._transform_maps(u.multiply_asym(P0[1], P0[0], Q_maps[1], Q_maps[0]),
                                                                 p, w)
                    Qs[3, ii] += 54. / 25. * self._transform_maps(u.multiply(P0[0], P0[1], P0[1]), q, w)
                if t == 'gNL-con':
                    w, f = self.r_weights[t], self.d_rlXs
                    R = R_maps
                    for k, (i, j, l) in enumerate(((0, 0, 0), (1, 1, 1), (0, 0, 1), (0, 1, 1))):
                        Qs[k, ii] = 216. / 25. * self._transform_maps(self.utils.multiply(R[i], R[j], R[l]), f, w)
                if t == 'gNL-dotdot':
                    w = self.rtau_weights[t]
                    f = self.d_alXs * self._tau_pow(4)
                    A = A_maps
                    for k, (i, j, l) in enumerate(((0, 0, 0), (1, 1, 1), (0, 0, 1), (0, 1, 1))):
                        Qs[k, ii] = 9216. / 25. * self._transform_maps(self.utils.multiply(A[i], A[j], A[l]), f, w)
                if t == 'tauNL-loc':
                    w = self.r_weights[t]
                    F_vecs = self._F_PQ(P_maps[0], Q_maps, w)
                    Qs[:, ii] += (4. * np.pi) ** 1.5 * self._get_Q4_perms(P_maps[0], Q_maps, F_vecs, w)
                    del F_vecs
                if _is_direc(t):
                    w = self.r_weights[t]
                    # polyspec/tspec_template.py:2850-2893: n1 != n3 adds both orderings, symmetrised
                    parts = []
                    for n1, n3, n, wp in self._direc_parts(t):
                        parts += ([(n1, n3, n, wp)] if n1 == n3 else
                                  [(n1, n3, n, 0.5 * wp), (n3, n1, n, 0.5 * (-1.) ** (n1 + n3) * wp)])
                    for a, c, n, wt in parts:
                        if a == 0 and c == 0:
                            F_vecs = self._F_PQ(P_maps[0], Q_maps, w)
                            Qs[:, ii] += wt * self._get_Q4_perms(P_maps[0], Q_maps, F_vecs, w)
                        elif a == 0:
                            # the n1 = 0 rows read the real part of the mu1 = 0 F maps (ideal_fisher.pyx:177, :325)
                            F_vecs = self._F_PQ_n(P_maps[c], Q_maps, w, a, c, n)
                            Qs[:, ii] += wt * self._get_Q4_perms(P_maps[0], Q_maps, F_vecs[:, 0].real.contiguous(), w)
                        else:
                            F_vecs = self._F_PQ_n(P_maps[c], Q_maps, w, a, c, n)
                            Qs[:, ii] += wt * self._get_Q4_perms_n(P_maps[a], Q_maps, F_vecs, w, a)
                        del F_vecs
                if _is_coll(t):
                    # collider Q-derivative (polyspec/tspec_template.py:2691-2706, 2896-2914)
                    w = self.r_weights[t]
                    s_, x = _coll_parse(t)
                    beta = -1.5 + x if 'tauNL-light' in t else -1.5 - 1.0j * x
                    Ps = coll_P[beta, s_]
                    cPs = coll_P[np.conj(beta), s_] if np.imag(beta) != 0 else None
                    F_vecs = self._coll_F_PQ(Ps, Q_maps, w, s_, beta, conjPs_maps=cPs)
                    Qs[:, ii] += self._get_Q4_perms_coll(Ps, Q_maps, F_vecs, w, s_, beta, cPs)
                    del F_vecs
                if t == 'gNL-dotdel':
                    Qs[:, ii] = self._dotdel_Q(A_maps, B_maps, C_maps, self.rtau_weights[t])
                if t == 'gNL-deldel':
                    Qs[:, ii] = self._deldel_Q(B_maps, C_maps, self.rtau_weights[t])
                if t == 'lensing':
                    Qs[:, ii] += self._lensing_Q(U_maps, V_maps)
                if t == 'point-source':
                    u0 = U_maps[:, 0]

                    def psq(m):
                        q = torch.zeros((1 + 2 * self.pol, len(self.ls)), dtype=torch.complex128, device=self._dev)
                        q[0] = b.to_lm(m.real[None], lmax=self.lmax)[0, self.d_lminfilt]
                        return q
                    Qs[0, ii] = psq(u0[0] ** 3)
                    Qs[1, ii] = psq(u0[1] ** 3)
                    Qs[2, ii] = psq(u0[0] ** 2 * u0[1])
                    Qs[3, ii] = psq(u0[1] ** 2 * u0[0])
            flat = Qs.reshape(4 * nt, 1 + 2 * self.pol, len(self.ls))
            flat = self._weight_Q_maps(flat, weighting)
            return flat.reshape(4, nt, -1)

        Q4_Sinv = compute_Q4('Sinv')
        Q4_Ainv = compute_Q4('Ainv')
        t0 = time.time()
        fish = pixel.outer_product(Q4_Sinv, Q4_Ainv, self.base.nthreads, False)
        self._timed('fish_outer', t0)
        self.timers['fisher'] += time.time() - t_start
        return fish.cpu().numpy()

    def compute_fisher(self, N_it, verb=False):
        """Monte Carlo Fisher matrix over seeds 0..N_it-1 (polyspec/tspec_template.py:3054-3072)."""
        fish = np.zeros((len(self.templates), len(self.templates)))
        for seed in range(N_it):
            print("Computing Fisher contribution %d of %d" % (seed + 1, N_it))
            fish += self.compute_fisher_contribution(seed, verb=verb * (seed == 0)) / N_it
        self.fish = fish
        self.inv_fish = np.linalg.inv(fish)
        return fish

    def Tl_unwindowed(self, data, fish=[], include_disconnected_term=True, verb=False, input_type='map'):
        """inv(F) times the numerator, one entry per template (polyspec/tspec_template.py:3074-3108)."""
        if len(fish) != 0:
            self.fish = fish
            self.inv_fish = np.linalg.inv(fish)
        if not hasattr(self, 'inv_fish'):
            raise Exception("Need to compute Fisher matrix first!")
        Tl_num = self.Tl_numerator(data, verb=verb, include_disconnected_term=include_disconnected_term,
                                   input_type=input_type)
        Tl_out = np.matmul(self.inv_fish, Tl_num)
        return {t: Tl_out[i] for i, t in enumerate(self.templates)}

    def optimize_radial_sampling_1d(self, *args, **kwargs):
        raise NotImplementedError("the radial-sampling optimiser is not implemented by the CUDA backend")

    def optimize_radial_sampling_2d(self, *args, **kwargs):
        raise NotImplementedError("the radial-sampling optimiser is not implemented by the CUDA backend")
