"""Binned bispectrum estimator on the GPU (mirror of polyspec/bspec_bin.py).

``BSpecBin(base, mask, applySinv, l_bins, l_bins_squeeze=[],
include_partial_triangles=False, fields=[...], parity='both')`` keeps the
reference interface, its bin list (``all_bins``, same order), symmetry factors,
``get_ells``, simulation handling (``generate_sims``, ``load_sims``) and
estimator methods (``Bl_numerator``, ``compute_fisher_contribution``,
``compute_fisher``, ``Bl_unwindowed``, ``Bl_numerator_ideal``,
``compute_fisher_ideal``, ``Bl_ideal``).
``applySinv`` receives and returns CUDA tensors (maps ``float64 [nfield, Npix]``,
alm ``complex128 [nfield, nlm]``); an ``applySinv`` with a ``.batched`` method (a
callable on a leading batch axis, e.g. ``Weightings.make_applySinv``) filters the
Q3 rows of the Fisher contribution in batches.

How the work maps to the device:

* H maps.  Every ``compute_spin_transform_map`` of one harmonic field over all
  l-bins and used fields (polyspec/bspec_bin.py:177-184, :330-331) is one
  batched spin-1 and one batched spin-2 synthesis of the inputs (G, C) = (-a, 0);
  the plus map is G_map + i C_map and the minus map its complex conjugate times
  (-1)^s, so the maps are kept as the synthesis wrote them (planar real and
  imaginary planes).
* Triplet sums.  All pixel sums of ``Bl_numerator`` (:339-364, :383-415) and
  ``Bl_numerator_ideal`` run as one ``ps_bispec_triplet_sums`` launch per data set
  (the cubic term) and per simulation (the linear term).
* Q3 maps.  For a pair of H maps the reference forms
  to_lm_spin(H+1 H+1, H-1 H-1, 2) and the spin-1 cross terms (:496-518).  Both have
  minus map = conj(plus map), so each is one adjoint transform of (Re P, Im P),
  and the two spin-1 cross terms (or twice the one, on the diagonal) add in pixel
  space before a single spin-1 adjoint.  With (G2, C2), (G1, C1) the adjoint
  outputs, the row combinations of :532-546 reduce to
  HH0 + HH1 = 2 (conj G1 - conj G2) and i (HH0 - HH1) = 2 (conj C1 + conj C2),
  so a Q3 row is a real combination of those per-pair vectors over its three
  (pair, field, l-bin) contributions, assembled by ``ps_bispec_assemble_q``.  The
  pair value is symmetric in its two H maps, so each unordered pair is
  transformed once.
* Fisher.  The four outer products of :577-582 equal one product of the
  differences, Re(conj(Q_S0 - Q_S1) (Q_A0 - Q_A1)^T) / 24, computed as one real
  GEMM over (Re, Im).
* Ideal Fisher.  The 3j-symbol sums of :699-827 as Gauss-Legendre quadratures of
  binned Wigner d-sums (see ``compute_fisher_ideal``).
"""
import ctypes

import numpy as np
import torch

from . import _lib

ALL_FIELDS = ['TTT', 'TTE', 'TEE', 'EEE', 'TBB', 'EBB', 'TTB', 'TEB', 'EEB', 'BBB']


def _vp(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


class BSpecBin:
    def __init__(self, base, mask, applySinv, l_bins, l_bins_squeeze=[], include_partial_triangles=False,
                 fields=ALL_FIELDS, parity='both'):
        self.base = base
        self.mask = mask
        self.applySinv = applySinv
        self.l_bins = l_bins
        self.pol = self.base.pol
        self.parity = parity
        self.fields = fields
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

        self.include_partial_triangles = include_partial_triangles
        self.beam = self.base.beam
        self.beam_lm = self.base.beam_lm

        for f in fields:
            assert f in ALL_FIELDS, "Unknown field '%s' supplied!" % f
        assert len(fields) == len(np.unique(fields)), "Duplicate fields supplied!"
        if not self.pol and fields != ['TTT']:
            print("## Polarization mode not turned on; setting fields to TT only!")
            self.fields = ['TTT']

        assert parity in ['even', 'odd', 'both'], "Parity must be one of 'even', 'odd' or 'both'!"
        if not self.pol and parity != 'even':
            print("Caution: scalar 3-point functions can't probe parity-odd primordial physics!")
        self.chi_arr = {'even': [1], 'odd': [-1], 'both': [1, -1]}[parity]

        if np.max(self.l_bins_squeeze) > base.lmax:
            raise Exception("Maximum l is larger than HEALPix resolution!")
        if np.max(self.l_bins) > base.lmax // 2:
            print("## Caution: Maximum l is greater than HEALPix-lmax/2; this might cause boundary effects.")
        print("Binning: %d bins in [%d, %d]" % (self.Nl, self.min_l, np.max(self.l_bins)))
        if self.Nl_squeeze != self.Nl:
            print("Squeezed binning: %d bins in [%d, %d]" % (self.Nl_squeeze, self.min_l, np.max(self.l_bins_squeeze)))

        self.ell_bins = [(self.base.l_arr >= self.l_bins_squeeze[b]) & (self.base.l_arr < self.l_bins_squeeze[b + 1])
                         for b in range(self.Nl_squeeze)]

        if np.std(self.mask) < 1e-12 and np.abs(np.mean(self.mask) - 1) < 1e-12:
            print("Mask: ones")
            self.ones_mask = True
        else:
            print("Mask: spatially varying")
            self.ones_mask = False

        # bin list in the reference's order (polyspec/bspec_bin.py:95-115)
        self.all_bins = []
        self.good_bins = []
        for u in self.fields:
            u1, u2, u3 = [self.base.indices[u[i]] for i in range(3)]
            p_u = int(np.prod([self.base.parities[u[i]] for i in range(3)]))
            for bin1 in range(self.Nl_squeeze):
                for bin2 in range(self.Nl_squeeze):
                    if u1 == u2 and bin2 < bin1:
                        continue
                    for bin3 in range(self.Nl_squeeze):
                        if u2 == u3 and bin3 < bin2:
                            continue
                        if not self._check_bin(bin1, bin2, bin3):
                            continue
                        if min([bin1, bin2, bin3]) >= self.Nl:
                            continue
                        self.all_bins.append([u1, u2, u3, bin1, bin2, bin3, p_u])
                        self.good_bins.append((bin1, bin2, bin3))
        self.all_bins = np.asarray(self.all_bins, dtype=np.int64).reshape(-1, 7)
        self._good = set(self.good_bins)
        self.is_good = lambda bins: tuple(int(b) for b in bins) in self._good

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
        """1 if the bin triplet obeys the triangle conditions (polyspec/bspec_bin.py:123-146)."""
        lb = self.l_bins_squeeze
        if self.include_partial_triangles:
            l1s = np.arange(lb[bin1], lb[bin1 + 1])[:, None, None]
            l2s = np.arange(lb[bin2], lb[bin2 + 1])[None, :, None]
            l3s = np.arange(lb[bin3], lb[bin3 + 1])[None, None, :]
            filt = (l3s >= abs(l1s - l2s)) * (l3s <= l1s + l2s)
            return 1 if np.sum(filt) > 0 else 0
        l1 = 0.5 * (lb[bin1] + lb[bin1 + 1])
        l2 = 0.5 * (lb[bin2] + lb[bin2 + 1])
        l3 = 0.5 * (lb[bin3] + lb[bin3 + 1])
        return 0 if (l3 < abs(l1 - l2) or l3 > l1 + l2) else 1

    def _compute_symmetry_factor(self):
        """Degeneracy of every bin, stacked over parities (polyspec/bspec_bin.py:148-175)."""
        self.sym_factor_all = []
        for chi in self.chi_arr:
            sym = []
            for u1, u2, u3, bin1, bin2, bin3, p_u in self.all_bins:
                if bin1 == bin2 and u1 == u2 and bin2 == bin3 and u2 == u3:
                    sym.append(6)
                elif (bin1 == bin2 and u1 == u2) or (bin2 == bin3 and u2 == u3):
                    sym.append(2)
                else:
                    sym.append(1)
            self.sym_factor_all.append(np.asarray(sym))
        self.sym_factor = np.concatenate(self.sym_factor_all)
        self.N_b = len(self.sym_factor)
        print("Using a total of %d bins" % self.N_b)

    def get_ells(self, field='TTT'):
        """Central (l1, l2, l3) of every bin of one field triplet (polyspec/bspec_bin.py:186-214)."""
        assert field in self.fields, "Specified field '%s' not in inputs!" % field
        u1, u2, u3 = [self.base.indices[field[i]] for i in range(3)]
        lb = self.l_bins_squeeze
        l1s, l2s, l3s = [], [], []
        for bin1 in range(self.Nl_squeeze):
            for bin2 in range(self.Nl_squeeze):
                if u1 == u2 and bin2 < bin1:
                    continue
                for bin3 in range(self.Nl_squeeze):
                    if u2 == u3 and bin3 < bin2:
                        continue
                    if not self.is_good([bin1, bin2, bin3]):
                        continue
                    if min([bin1, bin2, bin3]) >= self.Nl:
                        continue
                    l1s.append(0.5 * (lb[bin1] + lb[bin1 + 1]))
                    l2s.append(0.5 * (lb[bin2] + lb[bin2 + 1]))
                    l3s.append(0.5 * (lb[bin3] + lb[bin3 + 1]))
        return l1s, l2s, l3s

    # ------------------------------------------------------------------ device tables
    def _build_tables(self):
        if self._tables is not None:
            return self._tables
        if not hasattr(self, 'sym_factor'):
            self._compute_symmetry_factor()
        dev = self.base.device
        ab = self.all_bins
        n_all = len(ab)
        us = sorted(set(int(u) for u in ab[:, :3].ravel())) if n_all else [0]
        hpos = {u: i for i, u in enumerate(us)}
        nfu = len(us)
        nH = self.Nl_squeeze * nfu
        hid = lambda u, b: int(b) * nfu + hpos[int(u)]

        # numerator terms: P = +1 maps, M = -2 maps (polyspec/bspec_bin.py:349-351, :392-402)
        cubic, lin = [], []
        for u1, u2, u3, b1, b2, b3, p_u in ab:
            P = [hid(u1, b1), hid(u2, b2), hid(u3, b3)]
            M = [nH + p for p in P]
            Ps = [2 * nH + p for p in P]
            Ms = [3 * nH + p for p in P]
            cubic += [(P[0], P[1], M[2]), (P[1], P[2], M[0]), (P[2], P[0], M[1])]
            lin += [(P[0], Ps[1], Ms[2]), (P[1], Ps[2], Ms[0]), (P[2], Ps[0], Ms[1]),
                    (Ps[0], P[1], Ms[2]), (Ps[1], P[2], Ms[0]), (Ps[2], P[0], Ms[1]),
                    (Ps[0], Ps[1], M[2]), (Ps[1], Ps[2], M[0]), (Ps[2], Ps[0], M[1])]

        # Q3 pairs (unordered) and row contributions (polyspec/bspec_bin.py:468-547)
        pair_index = {}

        def pair(uA, bA, uB, bB):
            key = tuple(sorted([(int(uA), int(bA)), (int(uB), int(bB))]))
            if key not in pair_index:
                pair_index[key] = len(pair_index)
            return pair_index[key]

        contrib, coef = [], []
        for ci, chi in enumerate(self.chi_arr):
            for ii, (u1, u2, u3, b1, b2, b3, p_u) in enumerate(ab):
                which = 0 if p_u * chi == 1 else 1
                c = 2.0 / 3.0 / self.sym_factor[ii]
                contrib += [(pair(u1, b1, u2, b2), u3, b3, which),
                            (pair(u2, b2, u3, b3), u1, b1, which),
                            (pair(u1, b1, u3, b3), u2, b2, which)]
                coef += [c, c, c]
        pairs = sorted(pair_index.items(), key=lambda kv: kv[1])
        prods2, prods1 = [], []
        for (A, B), k in pairs:
            hA, hB = hid(*A), hid(*B)
            prods2.append((hA, hB, 0))                 # H+1_A H+1_B
            prods1 += [(hA, hB, 3), (hB, hA, 3)]       # -conj(H+1_A) H+2_B - conj(H+1_B) H+2_A
        npair = len(pairs)
        i32 = lambda x: torch.as_tensor(np.ascontiguousarray(np.asarray(x, dtype=np.int32)), device=dev)
        T = dict(
            us=us, nfu=nfu, nH=nH, n_all=n_all, npair=npair,
            cubic_ptr=i32(3 * np.arange(n_all + 1)), cubic=i32(np.asarray(cubic).reshape(-1, 3)),
            lin_ptr=i32(9 * np.arange(n_all + 1)), lin=i32(np.asarray(lin).reshape(-1, 3)),
            ptr2=i32(np.arange(npair + 1)), prods2=i32(np.asarray(prods2).reshape(-1, 3)),
            ptr1=i32(2 * np.arange(npair + 1)), prods1=i32(np.asarray(prods1).reshape(-1, 3)),
            row_ptr=i32(3 * np.arange(len(contrib) // 3 + 1)), contrib=i32(np.asarray(contrib).reshape(-1, 4)),
            coef=torch.as_tensor(np.asarray(coef, dtype=np.float64), device=dev),
            edges=i32(np.asarray(self.l_bins_squeeze)),
            l_of_lm=i32(self.base.l_arr),
            us_t=torch.as_tensor(us, device=dev),
        )
        self._tables = T
        return T

    # ------------------------------------------------------------------ device building blocks
    def _H_plus(self, a_lm, spins):
        """(+s)H maps of a_lm [nfield, nlm] for every l-bin and used field, as planar
        [nH, 2, Npix] real/imaginary planes (map index = bin * nfu + field position)."""
        T = self._build_tables()
        P = self.base.plan()
        a = a_lm[T['us_t']]                                             # [nfu, nlm]
        g = -(self.d_ell_bins[:, None, :] * a[None]).reshape(T['nH'], -1)
        x = torch.zeros((T['nH'], 2, a.shape[-1]), dtype=torch.complex128, device=a.device)
        x[:, 0] = g
        self.base.n_SHTs_reverse += T['nH'] * len(spins)
        return [P.synthesis(x, s) for s in spins]

    def _pm_maps(self, h_lm):
        """[(+1)H, (-2)H] of conj(h) for every bin and used field (polyspec/bspec_bin.py:330-331):
        planar [2 nH, 2, Npix]; (-2)H = conj((+2)H)."""
        p1, p2 = self._H_plus(torch.conj(h_lm), (1, 2))
        p2[:, 1].neg_()
        return torch.cat([p1, p2])

    def _triplet_sums(self, maps, ptr, terms):
        T = self._tables
        nmap = maps.shape[0]
        npix = maps.shape[-1]
        maps = maps.contiguous()
        nb = ctypes.c_size_t()
        _lib.call("ps_bispec_triplet_sums_workspace_bytes", nmap, npix, T['n_all'], ctypes.byref(nb))
        ws = torch.empty(max(int(nb.value), 16), dtype=torch.uint8, device=maps.device)
        out = torch.empty(T['n_all'], dtype=torch.complex128, device=maps.device)
        _lib.call("ps_bispec_triplet_sums", _vp(maps), nmap, npix, _vp(ptr), _vp(terms), T['n_all'], _vp(out),
                  _vp(ws), int(nb.value), _stream())
        return out

    def _reduce(self, S, chi_fixed=False):
        """Per-bin numerator from the complex triplet sums: A_pix Re(S or i S) / 3 / sym
        (polyspec/bspec_bin.py:356-364)."""
        S = S.cpu().numpy()
        n_all = len(self.all_bins)
        out = np.zeros(self.N_b)
        for full in range(self.N_b):
            idx = full % n_all
            chi = self.chi_arr[0 if chi_fixed else full // n_all]
            p_u = self.all_bins[idx, 6]
            v = S[idx].real if p_u * chi != -1 else -S[idx].imag
            out[full] = self.base.A_pix * v / 3. / self.sym_factor[idx]
        return out

    def _Q3(self, a_lm, weighting):
        """Q3 rows [N_b, nfield * nlm] for one GRF (polyspec/bspec_bin.py:441-568)."""
        T = self._build_tables()
        base = self.base
        P = base.plan()
        if weighting == 'Sinv':
            if self.ones_mask:
                U = self.applySinv(self.d_beam * a_lm, input_type='harmonic')
            else:
                U = self.applySinv(self.d_mask * base.to_map(self.d_beam * a_lm))
        else:
            U = base.applyAinv(a_lm, input_type='harmonic')
        Hp1, Hp2 = self._H_plus(U, (1, 2))
        npix, nlm = base.Npix, P.nalm
        npair = T['npair']
        A2 = torch.empty((npair, 2, nlm), dtype=torch.complex128, device=U.device)
        A1 = torch.empty_like(A2)
        scale = np.pi / (3. * base.Nside ** 2)
        chunk = max(1, min(npair, int(2 ** 31 // (16 * npix))))
        nH = T['nH']
        for k0 in range(0, npair, chunk):
            nc = min(chunk, npair - k0)
            X = torch.empty((nc, 2, npix), dtype=torch.float64, device=U.device)
            ptr2 = T['ptr2'][k0:]
            _lib.call("ps_bispec_pair_products", _vp(Hp1), nH, _vp(Hp1), nH, npix, _vp(ptr2), _vp(T['prods2']), nc,
                      _vp(X), _stream())
            A2[k0:k0 + nc] = P.adjoint(X, 2, scale)
            ptr1 = T['ptr1'][k0:]
            _lib.call("ps_bispec_pair_products", _vp(Hp1), nH, _vp(Hp2), nH, npix, _vp(ptr1), _vp(T['prods1']), nc,
                      _vp(X), _stream())
            A1[k0:k0 + nc] = P.adjoint(X, 1, scale)
            del X
        base.n_SHTs_forward += 2 * npair
        del Hp1, Hp2
        nf = len(self.d_beam)
        if weighting == 'Sinv':
            sc = self.d_mw[None].expand(nf, nlm).contiguous()
        else:
            sc = self.d_beam.contiguous()
        Q = torch.empty((self.N_b, nf, nlm), dtype=torch.complex128, device=U.device)
        _lib.call("ps_bispec_assemble_q", _vp(A2), _vp(A1), npair, nlm, _vp(T['l_of_lm']), _vp(T['edges']),
                  self.Nl_squeeze, _vp(T['row_ptr']), _vp(T['contrib']), _vp(T['coef']), self.N_b, nf, _vp(sc),
                  _vp(Q), _stream())
        del A2, A1
        if weighting == 'Sinv':
            return Q.reshape(self.N_b, -1)
        return self._filter_rows(Q).reshape(self.N_b, -1)

    def _filter_rows(self, Qb):
        """S^-1 P of beam-weighted rows [R, nfield, nlm] (polyspec/bspec_bin.py:549-556)."""
        base = self.base
        R, nf = Qb.shape[0], Qb.shape[1]
        if self.ones_mask:
            if hasattr(self.applySinv, 'batched_harmonic'):
                return self.applySinv.batched_harmonic(Qb)
            return torch.stack([self.applySinv(Qb[r], input_type='harmonic') for r in range(R)])
        out = None
        chunk = max(1, min(R, int(2 ** 31 // (8 * nf * base.Npix))))
        for r0 in range(0, R, chunk):
            maps = base.to_map_batch(Qb[r0:r0 + chunk])
            maps *= self.d_mask[None]
            if hasattr(self.applySinv, 'batched'):
                y = self.applySinv.batched(maps)
            else:
                y = torch.stack([self.applySinv(m) for m in maps])
            if out is None:
                out = torch.empty((R,) + tuple(y.shape[1:]), dtype=y.dtype, device=y.device)
            out[r0:r0 + len(y)] = y
            del maps, y
        return out

    def _data_in(self, data):
        d, _ = self.base._in(data, torch.float64)
        return d

    # ------------------------------------------------------------------ simulations
    def _process_sim(self, sim, input_type='map'):
        """(+1)H and (-2)H maps of one simulation (polyspec/bspec_bin.py:216-228), as one
        planar map set."""
        if input_type == 'map':
            s, _ = self.base._in(sim, torch.float64)
        else:
            s, _ = self.base._in(sim, torch.complex128)
        h = self.applySinv(s, input_type=input_type)
        return self._pm_maps(h)

    def load_sims(self, load_sim, N_sims, verb=False, input_type='map', preload=True):
        """Simulations for the linear term from a loader (polyspec/bspec_bin.py:230-260)."""
        self.N_it = N_sims
        print("Using %d Monte Carlo simulations" % self.N_it)
        if preload:
            self.preload = True
            self.pm_maps = []
            for ii in range(self.N_it):
                if verb:
                    print("Loading bias simulation %d of %d" % (ii + 1, self.N_it))
                self.pm_maps.append(self._process_sim(load_sim(ii), input_type=input_type))
        else:
            self.preload = False
            if verb:
                print("No preloading; simulations will be loaded and accessed at runtime.")
            self.load_sim_data = lambda ii: self._process_sim(load_sim(ii), input_type=input_type)

    def generate_sims(self, N_sim, Cl_input=[], b_input=None, add_B=False, remove_mean=True, verb=False,
                      preload=True):
        """GRF simulations for the linear term (polyspec/bspec_bin.py:262-309)."""
        self.N_it = N_sim
        print("Using %d Monte Carlo simulations" % self.N_it)
        if len(Cl_input) == 0:
            Cl_input = self.base.Cl_tot

        def make(ii):
            if self.ones_mask:
                alpha_lm = self.base.generate_data(int(1e5) + ii, Cl_input=Cl_input, deconvolve_beam=False,
                                                   b_input=b_input, add_B=add_B, remove_mean=remove_mean,
                                                   output_type='harmonic')
                return self._process_sim(alpha_lm, input_type='harmonic')
            alpha = self.base.generate_data(int(1e5) + ii, Cl_input=Cl_input, deconvolve_beam=False,
                                            b_input=b_input, add_B=add_B, remove_mean=remove_mean)
            alpha = self.d_mask * self.base._in(alpha, torch.float64)[0]
            return self._process_sim(alpha)

        if preload:
            self.preload = True
            self.pm_maps = []
            for ii in range(self.N_it):
                if verb:
                    print("Generating bias simulation %d of %d" % (ii + 1, self.N_it))
                self.pm_maps.append(make(ii))
        else:
            self.preload = False
            if verb:
                print("No preloading; simulations will be loaded and accessed at runtime.")
            self.load_sim_data = make

    # ------------------------------------------------------------------ optimal estimator
    def Bl_numerator(self, data, include_linear_term=True, verb=False):
        """Numerator of the unwindowed bispectrum estimator (polyspec/bspec_bin.py:312-420)."""
        if not hasattr(self, 'sym_factor'):
            self._compute_symmetry_factor()
        if (not hasattr(self, 'preload')) and include_linear_term:
            raise Exception("Need to generate or specify bias simulations!")
        T = self._build_tables()
        h_data_lm = self.applySinv(self._data_in(data), input_type='map')
        if verb:
            print("Computing H maps")
        maps = self._pm_maps(h_data_lm)
        b3_num = self._reduce(self._triplet_sums(maps, T['cubic_ptr'], T['cubic']))
        b1_num = np.zeros(self.N_b)
        if not include_linear_term:
            print("No linear correction applied!")
        else:
            for ii in range(self.N_it):
                if (ii + 1) % 5 == 0 and verb:
                    print("Computing b_1 piece from simulation %d" % (ii + 1))
                sim = self.pm_maps[ii] if self.preload else self.load_sim_data(ii)
                S = self._triplet_sums(torch.cat([maps, sim]), T['lin_ptr'], T['lin'])
                b1_num -= self._reduce(S) / self.N_it
        return b3_num + b1_num

    def compute_fisher_contribution(self, seed, verb=False, a_lms=None):
        """Fisher contribution of one pair of GRF simulations (polyspec/bspec_bin.py:422-584).

        ``a_lms`` (two beam-deconvolved harmonic fields) may replace the fields drawn
        from ``seed``."""
        if not hasattr(self, 'sym_factor'):
            self._compute_symmetry_factor()
        if verb:
            print("# Generating GRFs")
        if a_lms is None:
            a_lms = [self.base.generate_data(seed=seed + int((1 + ii) * 1e8), deconvolve_beam=True,
                                             output_type='harmonic') for ii in range(2)]
        a_lms = [self.base._in(a, torch.complex128)[0] for a in a_lms]
        if verb:
            print("\n# Computing Q3 map for S^-1 weighting")
        dQS = self._Q3(a_lms[0], 'Sinv')
        dQS -= self._Q3(a_lms[1], 'Sinv')
        if verb:
            print("\n# Computing Q3 map for A^-1 weighting")
        dQA = self._Q3(a_lms[0], 'Ainv')
        dQA -= self._Q3(a_lms[1], 'Ainv')
        if verb:
            print("\n# Assembling Fisher matrix\n")
        xs = torch.view_as_real(dQS).reshape(self.N_b, -1)
        xa = torch.view_as_real(dQA).reshape(self.N_b, -1)
        fish = (xs @ xa.T) / 24.
        return fish.cpu().numpy()

    def compute_fisher(self, N_it, verb=False):
        """Monte Carlo Fisher matrix over seeds 0..N_it-1 (polyspec/bspec_bin.py:586-606)."""
        if not hasattr(self, 'sym_factor'):
            self._compute_symmetry_factor()
        fish = np.zeros((self.N_b, self.N_b))
        for seed in range(N_it):
            print("Computing Fisher contribution %d of %d" % (seed + 1, N_it))
            fish += self.compute_fisher_contribution(seed, verb=verb * (seed == 0)) / N_it
        self.fish = fish
        self.inv_fish = np.linalg.inv(fish)
        return fish

    def _to_dict(self, Bl_out):
        out = {}
        index = 0
        chi_name = {1: '+', -1: '-'}
        for chi in self.chi_arr:
            for u in self.fields:
                n = len(self.get_ells(u)[0])
                out['%s' % u + '%s' % chi_name[chi]] = Bl_out[index:index + n]
                index += n
        return out

    def Bl_unwindowed(self, data, fish=[], include_linear_term=True, verb=False):
        """inv(F) times the numerator, as a dict per field and parity (polyspec/bspec_bin.py:608-643)."""
        if len(fish) != 0:
            self.fish = fish
            self.inv_fish = np.linalg.inv(fish)
        if not hasattr(self, 'inv_fish'):
            raise Exception("Need to compute Fisher matrix first!")
        Bl_num = self.Bl_numerator(data, include_linear_term=include_linear_term, verb=verb)
        return self._to_dict(np.matmul(self.inv_fish, Bl_num))

    # ------------------------------------------------------------------ ideal estimator
    def Bl_numerator_ideal(self, data, verb=False):
        """Ideal numerator normalised by <mask^3> (polyspec/bspec_bin.py:646-700).  The
        reference evaluates every bin with the first parity of ``chi_arr`` (its
        chi_index is taken after the modulo), which is kept."""
        if not hasattr(self, 'sym_factor'):
            self._compute_symmetry_factor()
        T = self._build_tables()
        d = self._data_in(data)
        Cinv = self.d_beam * torch.einsum('ijk,jk->ik', self.base.dev('inv_Cl_tot_lm_mat'), self.base.to_lm(d))
        maps = self._pm_maps(Cinv)
        out = self._reduce(self._triplet_sums(maps, T['cubic_ptr'], T['cubic']), chi_fixed=True)
        return out / np.mean(np.asarray(self.mask) ** 3)

    _PERMS = ((0, 1, 2), (1, 2, 0), (2, 0, 1), (0, 2, 1), (1, 0, 2), (2, 1, 0))

    def compute_fisher_ideal(self, verb=False, N_cpus=1):
        """Analytic ideal (unit-mask) Fisher matrix (polyspec/bspec_bin.py:699-827).

        The reference sums fac tj^2 x beams x (2l+1)^3 / (4 pi) x the six-permutation
        inverse-covariance product over every (l1, l2, l3) of each pair of bin triplets with
        equal sorted bins, with 3j symbols from pywigxjpf.  Here each permutation's sum is a
        product of three per-position factors h(l) = beam beam' Cinv (2l + 1), so it runs
        as Gauss-Legendre quadratures of binned Wigner d-sums (``ps_wigner_binned``,
        ``ps_bispec_ideal_contract``; the Gaunt identity Int d d d = 2 (3j)(3j)), split into
        even and odd l1 + l2 + l3 by (-1)^l factors.  The pair enumeration, the parity
        (real / imaginary part) selection and the symmetry-factor normalisation follow the
        reference; ``N_cpus`` has no counterpart."""
        if not hasattr(self, 'sym_factor'):
            self._compute_symmetry_factor()
        ab = np.asarray(self.all_bins)
        lb = np.asarray(self.l_bins_squeeze, dtype=np.int64)
        nbins, Lmax = len(lb) - 1, int(lb[-1]) - 1
        groups = {}
        for i, row in enumerate(ab):
            groups.setdefault(tuple(sorted(int(b) for b in row[3:6])), []).append(i)
        gid, tasks, task_entry, entries = {}, [], [], []
        for idxs in groups.values():
            for a, i in enumerate(idxs):
                for j in idxs[a:]:
                    u, b, up, bp = ab[i][:3], ab[i][3:6], ab[j][:3], ab[j][3:6]
                    for sg in self._PERMS:
                        if all(b[k] == bp[sg[k]] for k in range(3)):
                            gs = [gid.setdefault((int(u[k]), int(up[k]), int(up[sg[k]])), len(gid)) for k in range(3)]
                            tasks.append((gs[0], b[0], gs[1], b[1], gs[2], b[2]))
                            task_entry.append(len(entries))
                    entries.append((i, j))
        dev = self.base.device
        ls = np.arange(Lmax + 1, dtype=np.float64)
        beam = np.asarray(self.beam, dtype=np.float64)
        icov = np.asarray(self.base.inv_Cl_tot_mat, dtype=np.float64)
        H = np.zeros((max(len(gid), 1), Lmax + 1))
        for (a, b_, c), g in gid.items():
            H[g] = beam[a][:Lmax + 1] * beam[b_][:Lmax + 1] * icov[a, c][:Lmax + 1] * (2. * ls + 1.)
        nk = (3 * Lmax) // 2 + 2
        x = torch.empty(nk, dtype=torch.float64, device=dev)
        w = torch.empty_like(x)
        _lib.call("ps_gl_nodes", nk, _vp(x), _vp(w), _stream())
        d_H = torch.as_tensor(H, device=dev)
        d_edges = torch.as_tensor(lb.astype(np.int32), device=dev)
        G = H.shape[0]
        Phi = torch.zeros((G, nbins, 4, 2, nk), dtype=torch.float64, device=dev)
        _lib.call("ps_wigner_binned", _vp(x), nk, Lmax, _vp(d_edges), nbins, _vp(d_H), G, _vp(Phi), _stream())
        d_tasks = torch.as_tensor(np.asarray(tasks, dtype=np.int32).reshape(-1, 6), device=dev)
        S = torch.empty((len(tasks), 2), dtype=torch.float64, device=dev)
        _lib.call("ps_bispec_ideal_contract", _vp(Phi), _vp(w), nk, G, nbins, _vp(d_tasks), len(tasks), _vp(S),
                  _stream())
        S = S.cpu().numpy()
        value = np.zeros(len(entries), dtype=np.complex128)
        np.add.at(value, np.asarray(task_entry, dtype=np.int64),
                  ((S[:, 0] + S[:, 1]) / 2. + 1j * (S[:, 0] - S[:, 1]) / 2.) / (4. * np.pi))
        NB = self.N_b
        sym = np.asarray(self.sym_factor)
        fish = np.zeros((NB, NB))
        for e, (i, j) in enumerate(entries):
            pu, pup = ab[i][6], ab[j][6]
            for ci, chi in enumerate(self.chi_arr):
                for cj, chip in enumerate(self.chi_arr):
                    if pu * chi != pup * chip:
                        continue
                    out = value[e].real if pu * chi == 1 else value[e].imag
                    fish[ci * NB // 2 + i, cj * NB // 2 + j] = out / sym[i] / sym[j]
                    fish[cj * NB // 2 + j, ci * NB // 2 + i] = out / sym[i] / sym[j]
        if verb:
            print("Fisher matrix computation complete\n")
        self.fish_ideal = fish
        self.inv_fish_ideal = np.linalg.inv(self.fish_ideal)
        return fish

    def Bl_ideal(self, data, fish_ideal=[], verb=False, N_cpus=1):
        """Ideal estimator with a supplied ideal Fisher matrix (polyspec/bspec_bin.py:822-861)."""
        if len(fish_ideal) != 0:
            self.fish_ideal = fish_ideal
            self.inv_fish_ideal = np.linalg.inv(fish_ideal)
        if not hasattr(self, 'inv_fish_ideal'):
            print("Computing ideal Fisher matrix")
            self.compute_fisher_ideal(verb=verb, N_cpus=N_cpus)
        Bl_num_ideal = self.Bl_numerator_ideal(data, verb=verb)
        return self._to_dict(np.matmul(self.inv_fish_ideal, Bl_num_ideal))
