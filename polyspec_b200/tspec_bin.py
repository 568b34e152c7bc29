"""Binned trispectrum estimator on the GPU (mirror of polyspec/tspec_bin.py).

``TSpecBin(base, mask, applySinv, l_bins, l_bins_squeeze=[], L_bins=[],
include_partial_triangles=False, fields=[...], parity='both')`` keeps the
reference interface, its bin ordering, symmetry factors, ``get_ells``,
simulation handling (``generate_sims``, ``load_sims``) and the optimal estimator
(``Tl_numerator``, ``compute_fisher_contribution``, ``compute_fisher``,
``Tl_unwindowed``) and the ideal estimator's numerator (``Tl_numerator_ideal``,
with its 3j-symbol 0- and 2-field terms as Gauss-Legendre quadratures of binned
Wigner d-sums) and ``Tl_ideal`` with a supplied ideal Fisher matrix;
``compute_fisher_ideal`` (6j symbols) raises NotImplementedError.  ``applySinv`` receives and returns CUDA tensors; one with a
``.batched`` method filters the Fisher rows in batches.

How the work maps to the device (the algebra was checked on the CPU against the
reference to 1e-15 before the GPU code was written):

* H maps.  (+-1)H of bin b and field u (tspec_bin.py:235-242) is the spin-1
  synthesis of (G, C) = (-bin conj(h_u), 0): H+ = P = G_map + i C_map and
  H- = -conj(P); all bins and fields are one batched synthesis, kept planar.
* A fields (:244-277).  For a pair of H maps the reference's
  to_lm_spin(H+ H+', H- H-', 2)[::-1].conj() has minus map = conj(plus map), so
  it is one spin-2 adjoint of (Re X, Im X), X = P P' (or the symmetrised
  (P_a P'_b + P_b P'_a)/2 of two fields), with A = (-(conj G + i conj C),
  -(conj G - i conj C)).  Pair products run in ``ps_bispec_pair_products``, the
  adjoints as one batch; each unordered pair is transformed once.
* Numerator (:409-588).  Every summand is a binned m-weighted inner product
  Sum_{lm in L} m_w conj(X_1) Y_0 between two A fields; for each L bin these form
  the matrix (conj(X_1) w_L) Y_0^T over all pairs, one complex GEMM, from which
  the 4-, 2- and 0-field terms of every bin are gathered.
* Fisher (:590-817).  The binned A maps are spin-2 syntheses of (G bin_L, -C bin_L);
  each (H A) field of the reference is the spin-1 adjoint of -conj(P) A+ (minus
  map = conj(plus map)), and the reference's combinations of them for the four Q
  types (3 HA_111, 3 HA_222, 2 HA_112 + HA_211, 2 HA_212 + HA_122) are summed in
  pixel space before one adjoint each.  A Q4 row is then
  2/sym Sum (bin mask) conj(G1) or conj(C1) over its four (pair, partner)
  contributions -- conj(G1) where p_u chi = 1, conj(C1) otherwise -- written by
  ``ps_bispec_assemble_q`` with the m weights or the beam folded in; the A^-1 rows
  are filtered in batches; the Fisher matrix couples the four Q types with the
  reference's 4x4 weights as four real GEMMs.
"""
import ctypes

import numpy as np
import torch

from . import _lib

ALL_FIELDS = ['TTTT', 'TTTE', 'TTEE', 'TTBB', 'TETE', 'TEEE', 'TEBB', 'TBTB', 'TBEB', 'EEEE', 'EEBB', 'EBEB', 'BBBB',
              'TTTB', 'TTEB', 'TETB', 'TEEB', 'TBEE', 'TBBB', 'EEEB', 'EBBB']
# (multiplicity, H set, A variant) of the (H A) combinations of each Q type (tspec_bin.py:768-771)
_Q_TERMS = {0: [(3, 0, 0)], 1: [(3, 1, 1)], 2: [(2, 0, 2), (1, 1, 0)], 3: [(2, 1, 2), (1, 0, 1)]}


def _vp(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


class TSpecBin:
    def __init__(self, base, mask, applySinv, l_bins, l_bins_squeeze=[], L_bins=[], include_partial_triangles=False,
                 fields=ALL_FIELDS, parity='both'):
        self.base = base
        self.mask = mask
        self.applySinv = applySinv
        self.l_bins = l_bins
        self.pol = self.base.pol
        self.fields = fields
        self.parity = parity
        self.min_l = np.min(l_bins)
        self.Nl = len(l_bins) - 1
        if len(l_bins_squeeze) > 0:
            self.l_bins_squeeze = l_bins_squeeze
            self.Nl_squeeze = len(l_bins_squeeze) - 1
            for l_edge in self.l_bins:
                assert l_edge in self.l_bins_squeeze, "Squeezed bins must contain all the unsqueezed bins!"
        else:
            self.l_bins_squeeze = np.array(self.l_bins).copy()
            self.Nl_squeeze = self.Nl
        if len(L_bins) > 0:
            self.L_bins = L_bins
            self.NL = len(L_bins) - 1
            for L_edge in self.L_bins:
                assert L_edge in self.l_bins_squeeze, "l-bins must contain all L-bins!"
        else:
            self.L_bins = np.array(self.l_bins).copy()
            self.NL = self.Nl
        self.include_partial_triangles = include_partial_triangles
        if self.include_partial_triangles:
            print("Including triangles partially satisfying the triangle conditions (in the lowest bin only)")
        self.beam = self.base.beam
        self.beam_lm = self.base.beam_lm
        for f in fields:
            assert f in ALL_FIELDS, "Unknown field '%s' supplied!" % f
        assert len(fields) == len(np.unique(fields)), "Duplicate fields supplied!"
        assert parity in ['even', 'odd', 'both'], "Parity must be one of 'even', 'odd' or 'both'!"
        self.chi_arr = {'even': [1], 'odd': [-1], 'both': [1, -1]}[parity]
        if np.max(self.l_bins_squeeze) > base.lmax:
            raise Exception("Maximum l is larger than HEALPix resolution!")
        if np.max(self.l_bins) > base.lmax // 2:
            print("## Caution: Maximum l is greater than HEALPix-lmax/2; this might cause boundary effects.")
        print("Binning: %d bins in [%d, %d]" % (self.Nl, self.min_l, np.max(self.l_bins)))
        if self.Nl_squeeze != self.Nl:
            print("Squeezed binning: %d bins in [%d, %d]" % (self.Nl_squeeze, self.min_l, np.max(self.l_bins_squeeze)))
        if self.NL != self.Nl_squeeze:
            print("L binning: %d bins in [%d, %d]" % (self.NL, self.min_l, np.max(self.L_bins)))
        if np.std(self.mask) < 1e-12 and np.abs(np.mean(self.mask) - 1) < 1e-12:
            print("Mask: ones")
            self.ones_mask = True
        else:
            print("Mask: spatially varying")
            self.ones_mask = False
        self.ell_bins = [(self.base.l_arr >= self.l_bins_squeeze[b]) & (self.base.l_arr < self.l_bins_squeeze[b + 1])
                         for b in range(self.Nl_squeeze)]
        dev = base.device
        self.d_mask = torch.as_tensor(np.asarray(mask, dtype=np.float64), device=dev)
        if self.d_mask.dim() == 1:
            self.d_mask = self.d_mask[None]
        self.d_beam = base.dev('beam_lm')
        self.d_mw = base.dev('m_weight')
        self.d_ell_bins = torch.as_tensor(np.vstack(self.ell_bins).astype(np.float64), device=dev)
        self._tables = None

    # ------------------------------------------------------------------ binning (reference logic)
    def _check_bin(self, bin1, bin2, bin3):
        """Triangle conditions on bin centres, or on all modes of the lowest bin (tspec_bin.py:110-136)."""
        lb = self.l_bins_squeeze
        if ((bin1 <= 0) or (bin2 <= 0) or (bin3 <= 0)) and self.include_partial_triangles:
            for l1 in range(lb[bin1], lb[bin1 + 1]):
                for l2 in range(lb[bin2], lb[bin2 + 1]):
                    for l3 in range(lb[bin3], lb[bin3 + 1]):
                        if abs(l1 - l2) <= l3 <= l1 + l2:
                            return 1
            return 0
        l1 = 0.5 * (lb[bin1] + lb[bin1 + 1])
        l2 = 0.5 * (lb[bin2] + lb[bin2 + 1])
        l3 = 0.5 * (lb[bin3] + lb[bin3 + 1])
        return 0 if (l3 < abs(l1 - l2) or l3 > l1 + l2) else 1

    def _iter_bins(self, u1, u2, u3, u4):
        """Bin quintuplets of one field quadruplet in the reference's order (tspec_bin.py:147-187)."""
        for bin1 in range(self.Nl_squeeze):
            for bin2 in range(self.Nl_squeeze):
                if u1 == u2 and bin2 < bin1:
                    continue
                if min([bin1, bin2]) >= self.Nl:
                    continue
                for bin3 in range(self.Nl_squeeze):
                    if u1 == u3 and u2 == u4 and bin3 < bin1:
                        continue
                    for bin4 in range(self.Nl_squeeze):
                        if u3 == u4 and bin4 < bin3:
                            continue
                        if u1 == u3 and u2 == u4 and bin1 == bin3 and bin4 < bin2:
                            continue
                        if min([bin3, bin4]) >= self.Nl:
                            continue
                        for binL in range(self.NL):
                            if not self._check_bin(bin1, bin2, binL):
                                continue
                            if not self._check_bin(bin3, bin4, binL):
                                continue
                            yield bin1, bin2, bin3, bin4, binL

    def _compute_symmetry_factor(self):
        """Degeneracy of every bin, stacked over parities and fields (tspec_bin.py:138-188)."""
        self.sym_factor_all = []
        for chi in self.chi_arr:
            for u in self.fields:
                u1, u2, u3, u4 = [self.base.indices[u[i]] for i in range(4)]
                sym_factor = []
                for bin1, bin2, bin3, bin4, binL in self._iter_bins(u1, u2, u3, u4):
                    if bin1 == bin2 and bin3 == bin4 and bin1 == bin3 and u1 == u2 and u3 == u4 and u1 == u3:
                        sym = 8
                    elif bin1 == bin2 and bin3 == bin4 and u1 == u2 and u3 == u4:
                        sym = 4
                    elif (bin1 == bin2 and u1 == u2) or (bin3 == bin4 and u3 == u4):
                        sym = 2
                    elif bin1 == bin3 and bin2 == bin4 and u1 == u3 and u2 == u4:
                        sym = 2
                    else:
                        sym = 1
                    sym_factor.append(sym)
                self.sym_factor_all.append(np.asarray(sym_factor))
        self.sym_factor = np.concatenate(self.sym_factor_all)
        self.N_t = len(self.sym_factor)
        print("Using a total of %d bins" % self.N_t)

    def get_ells(self, field='TTTT'):
        """Central (l1, l2, l3, l4, L) of every bin of one field quadruplet (tspec_bin.py:190-233)."""
        assert field in self.fields, "Specified field '%s' not in inputs!" % field
        u1, u2, u3, u4 = [self.base.indices[field[i]] for i in range(4)]
        lb, Lb = self.l_bins_squeeze, self.L_bins
        c = lambda e, b: 0.5 * (e[b] + e[b + 1])
        l1s, l2s, l3s, l4s, Ls = [], [], [], [], []
        for bin1, bin2, bin3, bin4, binL in self._iter_bins(u1, u2, u3, u4):
            l1s.append(c(lb, bin1))
            l2s.append(c(lb, bin2))
            l3s.append(c(lb, bin3))
            l4s.append(c(lb, bin4))
            Ls.append(c(Lb, binL))
        return l1s, l2s, l3s, l4s, Ls

    # ------------------------------------------------------------------ device tables
    def _build_tables(self):
        if self._tables is not None:
            return self._tables
        if not hasattr(self, 'sym_factor'):
            self._compute_symmetry_factor()
        dev = self.base.device
        quads = []
        for u in self.fields:
            u1, u2, u3, u4 = [self.base.indices[u[i]] for i in range(4)]
            p_u = int(np.prod([self.base.parities[u[i]] for i in range(4)]))
            for bins in self._iter_bins(u1, u2, u3, u4):
                quads.append((u1, u2, u3, u4) + tuple(bins) + (p_u,))
        quads = np.asarray(quads, dtype=np.int64).reshape(-1, 10)
        us = sorted(set(int(x) for x in quads[:, :4].ravel())) if len(quads) else [0]
        hpos = {u: i for i, u in enumerate(us)}
        nfu = len(us)
        nH = self.Nl_squeeze * nfu
        hid = lambda u, b: int(b) * nfu + hpos[int(u)]
        pair_index = {}

        def pair(i, j):
            key = (min(i, j), max(i, j))
            if key not in pair_index:
                pair_index[key] = len(pair_index)
            return pair_index[key]

        pA = np.array([pair(hid(q[0], q[4]), hid(q[1], q[5])) for q in quads], dtype=np.int64)
        pB = np.array([pair(hid(q[2], q[6]), hid(q[3], q[7])) for q in quads], dtype=np.int64)
        pairs = sorted(pair_index.items(), key=lambda kv: kv[1])
        i32 = lambda x: torch.as_tensor(np.ascontiguousarray(np.asarray(x, dtype=np.int32)), device=dev)
        one = [(i, j, 0) for (i, j), _ in pairs]
        two = []
        for (i, j), _ in pairs:
            two += [(i, nH + j, 0), (nH + i, j, 0)]
        T = dict(quads=quads, us=us, nfu=nfu, nH=nH, hid=hid, pA=pA, pB=pB, npair=len(pairs), pairs=pairs,
                 us_t=torch.as_tensor(us, device=dev),
                 ptr1=i32(np.arange(len(pairs) + 1)), prods1=i32(np.asarray(one).reshape(-1, 3)),
                 ptr2=i32(2 * np.arange(len(pairs) + 1)), prods2=i32(np.asarray(two).reshape(-1, 3)),
                 edges=i32(np.asarray(self.l_bins_squeeze)), l_of_lm=i32(self.base.l_arr),
                 Ls=sorted(set(int(x) for x in quads[:, 8])))
        self._tables = T
        return T

    # ------------------------------------------------------------------ building blocks
    def _P(self, h_lm):
        """P = (+1)H of conj(h) for every bin and used field: planar [nH, 2, Npix] (tspec_bin.py:235-242)."""
        T = self._build_tables()
        a = torch.conj(h_lm[T['us_t']])
        g = -(self.d_ell_bins[:, None, :] * a[None]).reshape(T['nH'], -1)
        x = torch.zeros((T['nH'], 2, a.shape[-1]), dtype=torch.complex128, device=a.device)
        x[:, 0] = g
        self.base.n_SHTs_reverse += T['nH']
        return self.base.plan().synthesis(x, 1)

    def _products(self, Aset, nA, Bset, nB, ptr, prods, n, k0):
        npix = self.base.Npix
        X = torch.empty((n, 2, npix), dtype=torch.float64, device=Aset.device)
        _lib.call("ps_bispec_pair_products", _vp(Aset), nA, _vp(Bset), nB, npix, _vp(ptr[k0:]), _vp(prods), n,
                  _vp(X), _stream())
        return X

    def _A(self, P1, P2=None):
        """(G, C) of every pair's A field [npair, 2, nlm] (tspec_bin.py:244-277)."""
        T = self._build_tables()
        b = self.base
        P = b.plan()
        npix, npair, nH = b.Npix, T['npair'], T['nH']
        out = torch.empty((npair, 2, P.nalm), dtype=torch.complex128, device=P1.device)
        scale = np.pi / (3. * b.Nside ** 2)
        if P2 is None:
            S, nS, ptr, prods = P1.contiguous(), nH, T['ptr1'], T['prods1']
        else:
            S, nS, ptr, prods = torch.cat([P1, P2]).contiguous(), 2 * nH, T['ptr2'], T['prods2']
        chunk = max(1, min(npair, int(2 ** 31 // (16 * npix))))
        for k0 in range(0, npair, chunk):
            n = min(chunk, npair - k0)
            out[k0:k0 + n] = P.adjoint(self._products(S, nS, S, nS, ptr, prods, n, k0), 2, scale)
        b.n_SHTs_forward += npair
        if P2 is not None:
            out *= 0.5
        return out

    @staticmethod
    def _A01(GC):
        Gb, Cb = torch.conj(GC[:, 0]), torch.conj(GC[:, 1])
        return -(Gb + 1j * Cb), -(Gb - 1j * Cb)

    def _gram(self, X, Y):
        """M[L][p, q] = Sum_{lm in bin L} m_w conj(X_1[p]) Y_0[q] for the L bins in use."""
        T = self._build_tables()
        x1 = torch.conj(X[1])
        y0t = Y[0].transpose(0, 1)
        out = {}
        for L in T['Ls']:
            w = (self.d_mw * self.d_ell_bins[L]).to(torch.complex128)
            out[L] = (x1 * w[None]) @ y0t
        return out

    def _terms(self, M_fn):
        """Per-bin values f(p, q) (both orders gathered) for every (quad, parity)."""
        T = self._build_tables()
        q = T['quads']
        out = np.zeros(len(self.sym_factor), dtype=np.complex128)
        nq = len(q)
        for L in T['Ls']:
            sel = np.nonzero(q[:, 8] == L)[0]
            if len(sel) == 0:
                continue
            v = M_fn(L, torch.as_tensor(T['pA'][sel], device=self.base.device),
                     torch.as_tensor(T['pB'][sel], device=self.base.device)).cpu().numpy()
            for ci in range(len(self.chi_arr)):
                out[ci * nq + sel] = v
        return out

    def _real_part(self, z):
        T = self._build_tables()
        q = T['quads']
        nq = len(q)
        out = np.zeros(len(z))
        for ci, chi in enumerate(self.chi_arr):
            zz = z[ci * nq:(ci + 1) * nq]
            odd = q[:, 9] * chi == -1
            out[ci * nq:(ci + 1) * nq] = np.where(odd, -zz.imag, zz.real)
        return out

    # ------------------------------------------------------------------ simulations
    def _process_sim(self, sim_pair, input_type='map'):
        """H and A fields of one simulation pair (tspec_bin.py:279-300)."""
        dt = torch.float64 if input_type == 'map' else torch.complex128
        ha = self.applySinv(self.base._in(sim_pair[0], dt)[0], input_type=input_type)
        hb = self.applySinv(self.base._in(sim_pair[1], dt)[0], input_type=input_type)
        Pa, Pb = self._P(ha), self._P(hb)
        return Pa, Pb, self._A(Pa), self._A(Pb), self._A(Pa, Pb)

    def _store(self, res):
        Pa, Pb, Aaa, Abb, Aab = res
        self.H_a_maps.append(Pa)
        self.H_b_maps.append(Pb)
        self.A_aa_lms.append(Aaa)
        self.A_bb_lms.append(Abb)
        self.A_ab_lms.append(Aab)

    def load_sims(self, load_sim_pair, N_pairs, verb=False, preload=True, input_type='map'):
        """Simulation pairs from a loader (tspec_bin.py:302-346)."""
        self.N_it = N_pairs
        print("Using %d pairs of Monte Carlo simulations" % self.N_it)
        if preload:
            self.preload = True
            self.A_aa_lms, self.A_bb_lms, self.A_ab_lms, self.H_a_maps, self.H_b_maps = [], [], [], [], []
            for ii in range(self.N_it):
                if ii % 5 == 0 and verb:
                    print("Processing bias simulation %d of %d" % (ii + 1, self.N_it))
                self._store(self._process_sim(load_sim_pair(ii), input_type=input_type))
        else:
            self.preload = False
            if verb:
                print("No preloading; simulations will be loaded and accessed at runtime.")
            self.load_sim_data = lambda ii: self._process_sim(load_sim_pair(ii), input_type=input_type)

    def generate_sims(self, N_pairs, Cl_input=[], preload=True, verb=False):
        """GRF simulation pairs for the disconnected terms (tspec_bin.py:348-405)."""
        self.N_it = N_pairs
        print("Using %d pairs of Monte Carlo simulations" % self.N_it)
        if len(Cl_input) == 0:
            Cl_input = self.base.Cl_tot
        b = self.base

        def make(ii):
            if self.ones_mask:
                alpha = b.generate_data(int(1e5) + ii, Cl_input=Cl_input, output_type='harmonic', deconvolve_beam=False)
                beta = b.generate_data(int(2e5) + ii, Cl_input=Cl_input, output_type='harmonic', deconvolve_beam=False)
                return self._process_sim([alpha, beta], input_type='harmonic')
            alpha = self.d_mask * b._in(b.generate_data(int(1e5) + ii, Cl_input=Cl_input, deconvolve_beam=False),
                                        torch.float64)[0]
            beta = self.d_mask * b._in(b.generate_data(int(2e5) + ii, Cl_input=Cl_input, deconvolve_beam=False),
                                       torch.float64)[0]
            return self._process_sim([alpha, beta])

        if preload:
            self.preload = True
            self.H_a_maps, self.H_b_maps, self.A_aa_lms, self.A_bb_lms, self.A_ab_lms = [], [], [], [], []
            for ii in range(self.N_it):
                if ii % 5 == 0 and verb:
                    print("Generating bias simulation pair %d of %d" % (ii + 1, self.N_it))
                self._store(make(ii))
        else:
            self.preload = False
            if verb:
                print("No preloading; simulations will be loaded and accessed at runtime.")
            self.load_sim_data = make

    # ------------------------------------------------------------------ optimal estimator
    def Tl_numerator(self, data, include_disconnected_term=True, verb=False):
        """Numerator of the unwindowed trispectrum estimator (tspec_bin.py:409-588)."""
        if not hasattr(self, 'sym_factor'):
            self._compute_symmetry_factor()
        if not hasattr(self, 'preload') and include_disconnected_term:
            raise Exception("Need to generate or specify bias simulations!")
        if hasattr(self, 't0_num') and include_disconnected_term:
            compute_t0 = False
            if verb:
                print("Using precomputed t0 term")
        else:
            compute_t0 = True
        self._build_tables()
        h = self.applySinv(self.base._in(data, torch.float64)[0], input_type='map')
        if verb:
            print("Computing H maps")
        Pd = self._P(h)
        if verb:
            print("Computing A_lm fields")
        Add = self._A01(self._A(Pd))
        Mdd = self._gram(Add, Add)
        t4 = self._real_part(self._terms(lambda L, p, q: (Mdd[L][p, q] + Mdd[L][q, p]) / 2.))
        if not include_disconnected_term:
            print("## No subtraction of (parity-conserving) disconnected terms performed!")
            return t4 / self.sym_factor
        t2 = np.zeros(len(self.sym_factor))
        t0 = np.zeros(len(self.sym_factor))
        for ii in range(self.N_it):
            if self.preload:
                Pa, Pb = self.H_a_maps[ii], self.H_b_maps[ii]
                GCaa, GCbb, GCab = self.A_aa_lms[ii], self.A_bb_lms[ii], self.A_ab_lms[ii]
            else:
                Pa, Pb, GCaa, GCbb, GCab = self.load_sim_data(ii)
            Aaa, Abb = self._A01(GCaa), self._A01(GCbb)
            s2 = 0.
            for Axx, Pxx in ((Aaa, Pa), (Abb, Pb)):
                Axd = self._A01(self._A(Pxx, Pd))
                M1, M2, M3 = self._gram(Add, Axx), self._gram(Axx, Add), self._gram(Axd, Axd)
                s2 = s2 + self._terms(lambda L, p, q: M1[L][p, q] + M2[L][q, p] + 4 * (M3[L][p, q] + M3[L][q, p])
                                      + M2[L][p, q] + M1[L][q, p])
            t2 -= self._real_part(s2) / self.N_it / 4.
            if compute_t0:
                Aab = self._A01(GCab)
                M1, M2, M3 = self._gram(Abb, Aaa), self._gram(Aaa, Abb), self._gram(Aab, Aab)
                s0 = self._terms(lambda L, p, q: M1[L][p, q] + M2[L][q, p] + 4 * (M3[L][p, q] + M3[L][q, p])
                                 + M2[L][p, q] + M1[L][q, p])
                t0 += self._real_part(s0) / self.N_it / 4.
        if compute_t0:
            self.t0_num = t0 / self.sym_factor
        return (t4 + t2) / self.sym_factor + self.t0_num

    def _Q4(self, weighting, a_lms):
        """The four Q4 row sets [4, N_t, nfield * nlm] of one weighting (tspec_bin.py:609-812)."""
        T = self._build_tables()
        b = self.base
        P = b.plan()
        dev = b.device
        if weighting == 'Sinv':
            if self.ones_mask:
                U = [self.applySinv(self.d_beam * a, input_type='harmonic') for a in a_lms]
            else:
                U = [self.applySinv(self.d_mask * b.to_map(self.d_beam * a)) for a in a_lms]
        else:
            U = [b.applyAinv(a, input_type='harmonic') for a in a_lms]
        P1, P2 = self._P(U[0]), self._P(U[1])
        GC = [self._A(P1), self._A(P2), self._A(P1, P2)]  # A variants 11, 22, 12
        F = self._fisher_tables()
        nH, npl = T['nH'], F['npl']
        # binned A maps of every (pair, L): spin-2 synthesis of (G bin_L, -C bin_L), variants 11, 22, 12
        bl = self.d_ell_bins[F['pl_L']]                                  # [npl, nlm]
        x = torch.empty((npl, 3, 2, P.nalm), dtype=torch.complex128, device=dev)
        for v in range(3):
            x[:, v, 0] = GC[v][F['pl_pair'], 0] * bl
            x[:, v, 1] = -GC[v][F['pl_pair'], 1] * bl
        Ap = P.synthesis(x.reshape(3 * npl, 2, P.nalm), 2)
        b.n_SHTs_reverse += 3 * npl
        del x, GC, bl
        Hs = torch.cat([P1, P2]).contiguous()
        nf = len(self.d_beam)
        sc = self.d_mw[None].expand(nf, P.nalm).contiguous() if weighting == 'Sinv' else self.d_beam.contiguous()
        scale = np.pi / (3. * b.Nside ** 2)
        Q4 = []
        for tau in range(4):
            nkey, d_ptr, d_prods = F['nkey'], F['ptrs'][F['nterm'][tau]], F['prods'][tau]
            HA = torch.empty((nkey, 2, P.nalm), dtype=torch.complex128, device=dev)
            chunk = max(1, min(nkey, int(2 ** 31 // (16 * b.Npix))))
            for k0 in range(0, nkey, chunk):
                n = min(chunk, nkey - k0)
                HA[k0:k0 + n] = P.adjoint(self._products(Hs, 2 * nH, Ap, 3 * npl, d_ptr, d_prods, n, k0), 1, scale)
            b.n_SHTs_forward += nkey
            Q = torch.empty((len(self.sym_factor), nf, P.nalm), dtype=torch.complex128, device=dev)
            _lib.call("ps_bispec_assemble_q", None, _vp(HA), nkey, P.nalm, _vp(T['l_of_lm']), _vp(T['edges']),
                      self.Nl_squeeze, _vp(F['rows']), _vp(F['contrib']), _vp(F['coef']), len(self.sym_factor), nf,
                      _vp(sc), _vp(Q), _stream())
            del HA
            if weighting == 'Ainv':
                Q = self._filter_rows(Q)
            Q4.append(Q.reshape(len(self.sym_factor), -1))
        return torch.stack(Q4)

    def _fisher_tables(self):
        """Index tables of the Fisher contribution, which depend on the binning only: the
        (pair, L) list of binned A maps, the (H A) fields (one per (pair, L) and partner
        H map) with the pair-product terms of each Q type, and the four contributions of
        every Q4 row (tspec_bin.py:641-773)."""
        T = self._build_tables()
        if 'fisher' in T:
            return T['fisher']
        dev = self.base.device
        q = T['quads']
        nq, nH, hid = len(q), T['nH'], T['hid']
        pl_index = {}
        for k in range(nq):
            for pr in (T['pA'][k], T['pB'][k]):
                pl_index.setdefault((int(pr), int(q[k, 8])), len(pl_index))
        pls = sorted(pl_index.items(), key=lambda kv: kv[1])
        keys, contrib, coef = {}, [], []
        for ci, chi in enumerate(self.chi_arr):
            for k in range(nq):
                u1, u2, u3, u4, b1, b2, b3, b4, L, p_u = (int(v) for v in q[k])
                row = ci * nq + k
                which = 0 if p_u * chi == 1 else 1
                c = 2.0 / self.sym_factor[row]
                for pr, f, bn, pu, pb in ((T['pA'][k], u3, b3, u4, b4), (T['pA'][k], u4, b4, u3, b3),
                                          (T['pB'][k], u1, b1, u2, b2), (T['pB'][k], u2, b2, u1, b1)):
                    key = (pl_index[(int(pr), L)], hid(pu, pb))
                    if key not in keys:
                        keys[key] = len(keys)
                    contrib.append((keys[key], f, bn, which))
                    coef.append(c)
        i32 = lambda a: torch.as_tensor(np.ascontiguousarray(np.asarray(a, dtype=np.int32)), device=dev)
        ordered = sorted(keys.items(), key=lambda kv: kv[1])
        prods = []
        for tau in range(4):
            pt = []
            for (pli, item), _ in ordered:
                for mult, hset, var in _Q_TERMS[tau]:
                    pt.append((hset * nH + item, 3 * pli + var, 1 | 2 | (mult << 2)))  # -mult conj(P) A+
            prods.append(i32(np.asarray(pt).reshape(-1, 3)))
        nterm = [len(_Q_TERMS[tau]) for tau in range(4)]
        F = dict(npl=len(pls), nkey=len(keys),
                 pl_pair=torch.as_tensor([pr for (pr, L), _ in pls], device=dev),
                 pl_L=torch.as_tensor([L for (pr, L), _ in pls], device=dev),
                 prods=prods, rows=i32(4 * np.arange(len(self.sym_factor) + 1)),
                 contrib=i32(np.asarray(contrib).reshape(-1, 4)),
                 coef=torch.as_tensor(np.asarray(coef, dtype=np.float64), device=dev))
        # term pointers per Q type (1 or 2 terms per (H A) field)
        F['ptrs'] = {n: i32(n * np.arange(len(keys) + 1)) for n in set(nterm)}
        F['nterm'] = nterm
        T['fisher'] = F
        return F

    def _filter_rows(self, Qb):
        """S^-1 P of beam-weighted rows [R, nfield, nlm] (tspec_bin.py:776-787)."""
        base = self.base
        R, nf = Qb.shape[0], Qb.shape[1]
        if self.ones_mask:
            return torch.stack([self.applySinv(Qb[r], input_type='harmonic') for r in range(R)])
        out = None
        chunk = max(1, min(R, int(2 ** 31 // (8 * nf * base.Npix))))
        for r0 in range(0, R, chunk):
            maps = base.to_map_batch(Qb[r0:r0 + chunk]) * self.d_mask[None]
            if hasattr(self.applySinv, 'batched'):
                y = self.applySinv.batched(maps)
            else:
                y = torch.stack([self.applySinv(m) for m in maps])
            if out is None:
                out = torch.empty((R,) + tuple(y.shape[1:]), dtype=y.dtype, device=y.device)
            out[r0:r0 + len(y)] = y
        return out

    def compute_fisher_contribution(self, seed, verb=False, a_lms=None):
        """Fisher contribution of one pair of GRFs (tspec_bin.py:590-817).

        ``a_lms`` (two beam-deconvolved harmonic fields) may replace the fields drawn
        from ``seed``."""
        if not hasattr(self, 'sym_factor'):
            self._compute_symmetry_factor()
        if a_lms is None:
            a_lms = [self.base.generate_data(seed=seed + int((1 + ii) * 1e9), deconvolve_beam=True,
                                             output_type='harmonic') for ii in range(2)]
        a_lms = [self.base._in(a, torch.complex128)[0] for a in a_lms]
        if verb:
            print("\n# Computing Q4 map for S^-1 weighting")
        QS = self._Q4('Sinv', a_lms)
        if verb:
            print("\n# Computing Q4 map for A^-1 weighting")
        QA = self._Q4('Ainv', a_lms)
        return self._outer(QS, QA).cpu().numpy()

    @staticmethod
    def _outer(QS, QA):
        """Re Sum_{pq} c_pq conj(QS_p) QA_q^T / 24 / 48 with the Q-type coupling c of
        tspec_bin.py:806-814 (the same as ideal_fisher.pyx's outer_product): the four
        combinations Sum_q c_pq QA_q are formed first, then each p is one real GEMM over
        (Re, Im) -- O(N_t^2 K) on the GEMM units instead of eight complex products."""
        c = ((1., 0., 0., -3.), (0., 1., -3., 0.), (0., -3., 9., 0.), (-3., 0., 0., 9.))
        n = QS.shape[1]
        fish = torch.zeros((n, n), dtype=torch.float64, device=QS.device)
        for p in range(4):
            Bp = sum(c[p][q] * QA[q] for q in range(4) if c[p][q] != 0.)
            fish += torch.view_as_real(QS[p]).reshape(n, -1) @ torch.view_as_real(Bp).reshape(n, -1).T
            del Bp
        return fish / 24. / 48.

    def compute_fisher(self, N_it, verb=False):
        """Monte Carlo Fisher matrix over seeds 0..N_it-1 (tspec_bin.py:819-842)."""
        if not hasattr(self, 'sym_factor'):
            self._compute_symmetry_factor()
        fish = np.zeros((self.N_t, self.N_t))
        for seed in range(N_it):
            print("Computing Fisher contribution %d of %d" % (seed + 1, N_it))
            fish += self.compute_fisher_contribution(seed, verb=verb * (seed == 0)) / N_it
        self.fish = fish
        self.inv_fish = np.linalg.inv(fish)
        return fish

    def Tl_unwindowed(self, data, fish=[], include_disconnected_term=True, verb=False):
        """inv(F) times the numerator, as a dict per field and parity (tspec_bin.py:844-881)."""
        if len(fish) != 0:
            self.fish = fish
            self.inv_fish = np.linalg.inv(fish)
        if not hasattr(self, 'inv_fish'):
            raise Exception("Need to compute Fisher matrix first!")
        Tl_num = self.Tl_numerator(data, verb=verb, include_disconnected_term=include_disconnected_term)
        Tl_out = np.matmul(self.inv_fish, Tl_num)
        out = {}
        index, config_index = 0, 0
        chi_name = {1: '+', -1: '-'}
        for chi in self.chi_arr:
            for u in self.fields:
                n = len(self.sym_factor_all[config_index])
                out['%s' % u + '%s' % chi_name[chi]] = Tl_out[index:index + n]
                index += n
                config_index += 1
        return out

    # ------------------------------------------------------------------ ideal estimator
    def _ideal_t0_t2(self, C):
        """The 0- and 2-field terms of the ideal estimator (polyspec/tspec_bin.py:883-1045) for the
        data's beam C^-1 harmonics C [nfield, nlm].

        For each (bin1, bin2, binL) the reference sums over l1, l2, L (triangles)
            (2L+1) (l1 l2 L; -1 -1 2)^2 (-1)^L (2l1+1)(2l2+1)(-1)^(l1+l2) / (4 pi) x field factors,
        the field factors being products of one function of l1 and one of l2 (the empirical and
        theory inverse spectra times beams).  By the Gaunt identity
        (l1 l2 L; -1 -1 2)^2 = 1/2 Int d^{l1}_{-1,-1} d^{l2}_{-1,-1} d^L_{2,2} dx, each sum is a
        Gauss-Legendre quadrature of three binned d-sums (``ps_wigner_binned``, ``ps_quad_triple``).
        The assembly into the quadruplet list follows the reference."""
        b = self.base
        dev = b.device
        nf = 1 + 2 * self.pol
        lb = np.asarray(self.l_bins_squeeze, dtype=np.int64)
        Lb = np.asarray(self.L_bins, dtype=np.int64)
        lmx, Lmx = int(lb[-1]) - 1, int(Lb[-1]) - 1
        nb, nL = len(lb) - 1, len(Lb) - 1
        # empirical inverse spectrum of the data (tspec_bin.py:887-895)
        l_idx = torch.as_tensor(b.l_arr, device=dev)
        keep = l_idx <= lmx
        beam = torch.as_tensor(np.asarray(self.beam, dtype=np.float64)[:, :lmx + 1], device=dev)
        ls = torch.arange(lmx + 1, dtype=torch.float64, device=dev)
        Ce = torch.zeros((nf, nf, lmx + 1), dtype=torch.float64, device=dev)
        for u1 in range(nf):
            for u2 in range(nf):
                sq = (0.5 * (C[u1] * torch.conj(C[u2]) + C[u2] * torch.conj(C[u1])) * self.d_mw).real
                Ce[u1, u2].index_add_(0, l_idx[keep], sq[keep])
                Ce[u1, u2] *= beam[u1] * beam[u2] / (2. * ls + 1.)
        Ib = torch.as_tensor(np.asarray(b.inv_Cl_tot_mat, dtype=np.float64)[:nf, :nf, :lmx + 1], device=dev) \
            * beam[:, None, :] * beam[None, :, :]
        H = torch.cat([Ib.reshape(nf * nf, -1), Ce.reshape(nf * nf, -1)]) * (2. * ls + 1.)[None]
        HL = (2. * torch.arange(Lmx + 1, dtype=torch.float64, device=dev) + 1.)[None].contiguous()
        nk = (2 * lmx + Lmx) // 2 + 2
        x = torch.empty(nk, dtype=torch.float64, device=dev)
        w = torch.empty_like(x)
        _lib.call("ps_gl_nodes", nk, _vp(x), _vp(w), _stream())
        G = H.shape[0]
        Phi = torch.zeros((G, nb, 4, 2, nk), dtype=torch.float64, device=dev)
        H = H.contiguous()
        d_lb = torch.as_tensor(lb.astype(np.int32), device=dev)
        _lib.call("ps_wigner_binned", _vp(x), nk, lmx, _vp(d_lb), nb, _vp(H), G, _vp(Phi), _stream())
        PhiL = torch.zeros((1, nL, 4, 2, nk), dtype=torch.float64, device=dev)
        d_Lb = torch.as_tensor(Lb.astype(np.int32), device=dev)
        _lib.call("ps_wigner_binned", _vp(x), nk, Lmx, _vp(d_Lb), nL, _vp(HL), 1, _vp(PhiL), _stream())
        # rows: slot 0 = (-1,-1) (l1, l2), slot 3 = (2,2) (L); par 1 = (-1)^l weights
        row = lambda g, bb, q, nbb: ((g * nbb + bb) * 4 + q) * 2 + 1
        I_of = lambda a_, b_, bb: row(a_ * nf + b_, bb, 0, nb)
        C_of = lambda a_, b_, bb: row(nf * nf + a_ * nf + b_, bb, 0, nb)
        triples = [(b1, b2, bL) for b1 in range(nb) for b2 in range(nb) for bL in range(nL)
                   if self._check_bin(b1, b2, bL)]
        fp = [(a_, b_) for a_ in range(nf) for b_ in range(nf)]
        tasks = []
        for b1, b2, bL in triples:
            rl = row(0, bL, 3, nL)
            for a_, b_ in fp:
                for c_, d_ in fp:
                    tasks += [(C_of(a_, b_, b2), I_of(c_, d_, b1), rl), (I_of(a_, b_, b2), C_of(c_, d_, b1), rl),
                              (I_of(a_, b_, b1), I_of(c_, d_, b2), rl)]
        d_tasks = torch.as_tensor(np.asarray(tasks, dtype=np.int32).reshape(-1, 3), device=dev)
        out = torch.empty(len(tasks), dtype=torch.float64, device=dev)
        A = Phi.reshape(-1, nk)
        _lib.call("ps_quad_triple", _vp(A), A.shape[0], _vp(A), A.shape[0], _vp(PhiL), PhiL.numel() // nk, _vp(w), nk,
                  _vp(d_tasks), len(tasks), _vp(out), _stream())
        o = out.cpu().numpy().reshape(len(triples), nf, nf, nf, nf, 3) / (8. * np.pi)
        t2s = {t: -(o[i, ..., 0] + o[i, ..., 1]) for i, t in enumerate(triples)}
        t0s = {t: o[i, ..., 2] for i, t in enumerate(triples)}
        # assembly (tspec_bin.py:955-1022)
        T = self._build_tables()
        q = T['quads']
        NT, nq = self.N_t, len(q)
        t2n, t0n = np.zeros(NT), np.zeros(NT)
        for index, (u1, u2, u3, u4, b1, b2, b3, b4, bL, p_u) in enumerate(q):
            if ((b1 == b3) * (b2 == b4) + (b1 == b4) * (b2 == b3)) == 0:
                continue
            if (p_u == -1 and self.parity == 'even') or (p_u == 1 and self.parity == 'odd'):
                continue
            v0 = v2 = 0.
            if b1 == b3 and b2 == b4:
                v2 += t2s[b1, b2, bL][u2, u4, u3, u1]
                v0 += t0s[b1, b2, bL][u3, u1, u4, u2]
            if b1 == b4 and b2 == b3:
                v2 += t2s[b1, b2, bL][u2, u3, u4, u1]
                v0 += t0s[b1, b2, bL][u4, u1, u3, u2]
            for ci, chi in enumerate(self.chi_arr):
                if p_u * chi == -1:
                    continue
                t2n[ci * NT // 2 + index] = v2
                t0n[ci * NT // 2 + index] = v0
        t2 = t2n / np.mean(np.asarray(self.mask) ** 2) / self.sym_factor
        t0 = t0n / self.sym_factor
        return t0, t2

    def Tl_numerator_ideal(self, data, verb=False, include_disconnected_term=True, N_cpus=4):
        """Numerator of the ideal (unit-mask) trispectrum estimator (polyspec/tspec_bin.py:1047-1129),
        normalised by <mask^4>: the 4-field term from the A fields of beam C^-1 Y^dagger data (the
        same binned Gram matrices as Tl_numerator) plus the 0- and 2-field terms of _ideal_t0_t2.
        ``N_cpus`` has no counterpart."""
        if not hasattr(self, 'sym_factor'):
            self._compute_symmetry_factor()
        self._build_tables()
        b = self.base
        d = b._in(data, torch.float64)[0]
        C = self.d_beam * torch.einsum('ijk,jk->ik', b.dev('inv_Cl_tot_lm_mat'), b.to_lm(d))
        if verb:
            print("\nComputing H maps")
        Pd = self._P(C)
        if verb:
            print("Computing A_lm fields")
        Add = self._A01(self._A(Pd))
        Mdd = self._gram(Add, Add)
        t4 = self._real_part(self._terms(lambda L, p, q: (Mdd[L][p, q] + Mdd[L][q, p]) / 2.))
        out = t4 / np.mean(np.asarray(self.mask) ** 4.) / self.sym_factor
        if not include_disconnected_term:
            print("## No subtraction of (parity-conserving) disconnected terms performed!")
            return out
        t0, t2 = self._ideal_t0_t2(C)
        self.t0_num_ideal = t0
        return out + t2 + t0

    def compute_fisher_ideal(self, *args, **kwargs):
        """Analytic ideal Fisher matrix (polyspec/tspec_bin.py:1131-1370): needs Wigner 6j symbols and is
        not computed here; pass ``fish_ideal`` to Tl_ideal."""
        raise NotImplementedError("the ideal trispectrum Fisher matrix needs Wigner 6j symbols (pywigxjpf in "
                                  "the reference); pass fish_ideal to Tl_ideal")

    def Tl_ideal(self, data, fish_ideal=[], verb=False, include_disconnected_term=True, N_cpus=1):
        """Ideal estimator inv(F_ideal) x numerator, as a dict per field and parity
        (polyspec/tspec_bin.py:1372-1406).  The ideal Fisher matrix (6j symbols) is not computed
        here: pass ``fish_ideal``."""
        if len(fish_ideal) != 0:
            self.fish_ideal = fish_ideal
            self.inv_fish_ideal = np.linalg.inv(fish_ideal)
        if not hasattr(self, 'inv_fish_ideal'):
            print("Computing ideal Fisher matrix")
            self.compute_fisher_ideal(verb=verb, N_cpus=N_cpus)
        Tl_num_ideal = self.Tl_numerator_ideal(data, verb=verb, include_disconnected_term=include_disconnected_term)
        Tl_out = np.matmul(self.inv_fish_ideal, Tl_num_ideal)
        out = {}
        index, config_index = 0, 0
        chi_name = {1: '+', -1: '-'}
        for chi in self.chi_arr:
            for u in self.fields:
                n = len(self.sym_factor_all[config_index])
                out['%s' % u + '%s' % chi_name[chi]] = Tl_out[index:index + n]
                index += n
                config_index += 1
        return out
