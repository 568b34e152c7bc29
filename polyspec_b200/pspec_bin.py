"""Binned power-spectrum estimator on the GPU (mirror of polyspec/pspec_bin.py).

``PSpecBin(base, mask, applySinv, l_bins, fields=[...])`` keeps the
reference interface.  ``applySinv`` receives CUDA tensors (maps
``float64 [nfield, Npix]`` or alm ``complex128 [nfield, nlm]``) and must
return CUDA tensors; the ``Weightings`` methods of this package do.  The
Fisher outer product ``0.5 Re(Q_S^* Q_A^T)`` (polyspec/pspec_bin.py:162) is
one complex GEMM on the device.

``compute_fisher_contribution(seed, verb=False, batched=False)``: with
``batched=True`` and an ``applySinv`` exposing ``.batched`` (a callable on a
leading batch axis, see ``Weightings.batched_applySinv_optimal``) the N_p
weighted maps are filtered in one batched call instead of N_p calls.
"""
import numpy as np
import torch


class PSpecBin:
    def __init__(self, base, mask, applySinv, l_bins, fields=['TT', 'TE', 'TB', 'EE', 'EB', 'EE']):
        self.base = base
        self.mask = mask
        self.applySinv = applySinv
        self.l_bins = l_bins
        self.min_l = np.min(l_bins)
        self.Nl = len(l_bins) - 1
        self.pol = self.base.pol
        self.beam_lm = self.base.beam_lm
        self.fields = fields

        for f in fields:
            assert f in ['TT', 'TE', 'TB', 'EE', 'EB', 'BB'], "Unknown field '%s' supplied!" % f
        assert len(fields) == len(np.unique(fields)), "Duplicate fields supplied!"
        self.N_p = len(self.fields) * self.Nl

        if not self.pol and fields != ['TT']:
            print("## Polarization mode not turned on; setting fields to TT only!")
            self.fields = ['TT']

        if np.max(self.l_bins) > base.lmax:
            raise Exception("Maximum l is larger than HEALPix resolution!")
        if np.max(self.l_bins) > base.lmax // 2:
            print("## Caution: Maximum l is greater than HEALPix-lmax/2; this might cause boundary effects.")
        print("Binning: %d bins in [%d, %d]" % (self.Nl, self.min_l, np.max(self.l_bins)))
        print("Fields: %s" % fields)

        self.ell_bins = [(self.base.l_arr >= self.l_bins[bin1]) & (self.base.l_arr < self.l_bins[bin1 + 1])
                         for bin1 in range(self.Nl)]
        self.all_ell_bins = np.vstack(self.ell_bins)

        if np.std(self.mask) < 1e-12 and np.abs(np.mean(self.mask) - 1) < 1e-12:
            print("Mask: ones")
            self.ones_mask = True
        else:
            print("Mask: spatially varying")
            self.ones_mask = False

        dev = base.device
        self.d_ell_bins = torch.as_tensor(self.all_ell_bins, device=dev)  # [Nl, nlm] bool
        self.d_mask = torch.as_tensor(np.asarray(mask, dtype=np.float64), device=dev)
        if self.d_mask.dim() == 1:
            self.d_mask = self.d_mask[None]
        self.d_beam = base.dev('beam_lm')
        self.d_mw = base.dev('m_weight')

    def get_ells(self):
        return [0.5 * (self.l_bins[bin1] + self.l_bins[bin1 + 1]) for bin1 in range(self.Nl)]

    # ---------------------------------------------------------------- optimal estimator
    def _binned_auto(self, h):
        """1/Delta2 sum_lm m_w conj(h_u1) h_u2 [bin]  for every field (polyspec/pspec_bin.py:78-90)."""
        out = []
        binsf = self.d_ell_bins.to(torch.float64)
        for u in self.fields:
            u1, u2 = self.base.indices[u[0]], self.base.indices[u[1]]
            Delta2_u = (u1 == u2) + 1.
            spec_squared = (torch.conj(h[u1]) * h[u2]).real * self.d_mw
            out.append((binsf @ spec_squared) / Delta2_u)
        return torch.stack(out)

    def Cl_numerator(self, data):
        """Numerator of the unwindowed power-spectrum estimator (polyspec/pspec_bin.py:70-92)."""
        d, as_torch = self.base._in(data, torch.float64)
        h_data_lm = self.applySinv(d, input_type='map')
        return self.base._out(self._binned_auto(h_data_lm), as_torch)

    def _Q2_rows(self, Uinv_a_lm):
        """The N_p summands  Uinv_a_lm_u * bin / Delta2  (polyspec/pspec_bin.py:126-141)."""
        rows = []
        binsf = self.d_ell_bins.to(torch.float64)
        for u in self.fields:
            u1, u2 = self.base.indices[u[0]], self.base.indices[u[1]]
            Delta2_u = (u1 == u2) + 1.
            U = torch.zeros_like(Uinv_a_lm)
            U[u1] += Uinv_a_lm[u2]
            U[u2] += Uinv_a_lm[u1]
            for bin1 in range(self.Nl):
                rows.append(U * binsf[bin1] / Delta2_u)
        return rows

    def compute_fisher_contribution(self, seed, verb=False, batched=False, rng='numpy', a_lm=None):
        """Fisher contribution of one GRF simulation (polyspec/pspec_bin.py:94-164).

        ``a_lm`` (beam-deconvolved GRF harmonics) may be passed in place of the
        simulation drawn from ``seed``.
        """
        if verb:
            print("Generating GRF")
        if a_lm is None:
            a_lm = self.base.generate_data(seed=seed + int(1e7), output_type='harmonic', deconvolve_beam=True, rng=rng)
        a_lm, _ = self.base._in(a_lm, torch.complex128)

        if batched and not self.ones_mask and hasattr(self.applySinv, 'batched'):
            # the S^-1 solve of the simulation and the N_p solves of the Q_A rows are
            # independent: one batched solve of N_p + 1 right-hand sides
            Uinv_A = self.base.applyAinv(a_lm, input_type='harmonic')
            rows = self._Q2_rows(Uinv_A)
            alms = torch.stack([self.d_beam * a_lm] + [self.d_beam * r for r in rows])
            maps = self.d_mask[None] * self.base.to_map_batch(alms)
            sol = self.applySinv.batched(maps)
            Uinv_S = sol[0]
            Q_S = torch.stack([(self.d_mw * r).reshape(-1) for r in self._Q2_rows(Uinv_S)])
            Q_A = sol[1:].reshape(len(rows), -1)
            fish = 0.5 * torch.real(Q_S.conj() @ Q_A.T)
            return fish.cpu().numpy()

        # S^-1 weighting: Q_S rows are m_w * summand
        if self.ones_mask:
            Uinv_S = self.applySinv(self.d_beam * a_lm, input_type='harmonic')
        else:
            Uinv_S = self.applySinv(self.d_mask * self.base.to_map(self.d_beam * a_lm))
        Q_S = torch.stack([(self.d_mw * r).reshape(-1) for r in self._Q2_rows(Uinv_S)])

        # A^-1 weighting: Q_A rows are S^-1 P (beam * summand)
        Uinv_A = self.base.applyAinv(a_lm, input_type='harmonic')
        rows = self._Q2_rows(Uinv_A)
        if self.ones_mask:
            Q_A = torch.stack([self.applySinv(self.d_beam * r, input_type='harmonic').reshape(-1) for r in rows])
        else:
            Q_A = torch.stack([self.applySinv(self.d_mask * self.base.to_map(self.d_beam * r)).reshape(-1)
                               for r in rows])
        if verb:
            print("Assembling Fisher matrix\n")
        fish = 0.5 * torch.real(Q_S.conj() @ Q_A.T)
        return fish.cpu().numpy()

    def compute_fisher_contributions(self, seeds, verb=False, rng='numpy', a_lms=None):
        """Fisher contributions [K, N_p, N_p] of K GRF simulations (seeds, or beam-deconvolved harmonics
        a_lms), each as compute_fisher_contribution (polyspec/pspec_bin.py:94-164), with one batched S^-1
        solve of all K (N_p + 1) right-hand sides.  The systems are independent and each keeps its own
        stopping test, so the solve of the union is the solves of the parts; batching the simulations
        shares the last CG steps, which few systems of each simulation still take, between them."""
        K = len(a_lms) if a_lms is not None else len(seeds)
        if self.ones_mask or not hasattr(self.applySinv, 'batched'):
            return np.stack([self.compute_fisher_contribution(None if seeds is None else seeds[k], verb=verb,
                                                              batched=True, rng=rng,
                                                              a_lm=None if a_lms is None else a_lms[k])
                             for k in range(K)])
        alms, nrows = [], []
        for k in range(K):
            if a_lms is None:
                a_lm = self.base.generate_data(seed=seeds[k] + int(1e7), output_type='harmonic',
                                               deconvolve_beam=True, rng=rng)
            else:
                a_lm = a_lms[k]
            a_lm, _ = self.base._in(a_lm, torch.complex128)
            rows = self._Q2_rows(self.base.applyAinv(a_lm, input_type='harmonic'))
            alms.append(torch.stack([self.d_beam * a_lm] + [self.d_beam * r for r in rows]))
            nrows.append(len(rows))
        maps = self.d_mask[None] * self.base.to_map_batch(torch.cat(alms))
        del alms
        sol = self.applySinv.batched(maps)
        del maps
        out, o = [], 0
        for k in range(K):
            s = sol[o:o + nrows[k] + 1]
            o += nrows[k] + 1
            Q_S = torch.stack([(self.d_mw * r).reshape(-1) for r in self._Q2_rows(s[0])])
            Q_A = s[1:].reshape(nrows[k], -1)
            out.append(0.5 * torch.real(Q_S.conj() @ Q_A.T))
        return torch.stack(out).cpu().numpy()

    def compute_fisher(self, N_it, verb=False):
        """Monte Carlo Fisher matrix over seeds 0..N_it-1 (polyspec/pspec_bin.py:166-179)."""
        fish = np.zeros((self.N_p, self.N_p))
        for seed in range(N_it):
            print("Computing Fisher contribution %d of %d" % (seed + 1, N_it))
            fish += self.compute_fisher_contribution(seed, verb=verb) / N_it
        self.fish = fish
        self.inv_fish = np.linalg.inv(fish)
        return fish

    def Cl_unwindowed(self, data, fish=[]):
        """Unwindowed estimator inv(F) numerator (polyspec/pspec_bin.py:181-204)."""
        if len(fish) != 0:
            self.fish = fish
            self.inv_fish = np.linalg.inv(fish)
        if not hasattr(self, 'inv_fish'):
            raise Exception("Need to compute Fisher matrix first!")
        Cl_num = np.concatenate(np.asarray(self.Cl_numerator(np.asarray(data) if not isinstance(data, torch.Tensor) else data.cpu().numpy())))
        Cl_out = np.matmul(self.inv_fish, Cl_num)
        Cl_dict = {}
        index = 0
        for u in self.fields:
            Cl_dict['%s' % u] = Cl_out[index:index + self.Nl]
            index += self.Nl
        return Cl_dict

    # ---------------------------------------------------------------- ideal estimator
    def Cl_numerator_ideal(self, data):
        """Ideal numerator normalised by <mask^2> (polyspec/pspec_bin.py:207-228)."""
        d, as_torch = self.base._in(data, torch.float64)
        Cinv = self.d_beam * torch.einsum('ijk,jk->ik', self.base.dev('inv_Cl_tot_lm_mat'), self.base.to_lm(d))
        out = self._binned_auto(Cinv) / float(np.mean(np.asarray(self.mask) ** 2))
        return self.base._out(out, as_torch)

    def compute_fisher_ideal(self):
        """Analytic Fisher matrix of the ideal estimator (polyspec/pspec_bin.py:230-260)."""
        fish = np.zeros((len(self.fields) * self.Nl, len(self.fields) * self.Nl))
        icov = self.base.inv_Cl_tot_lm_mat
        for i, u in enumerate(self.fields):
            u1, u2 = self.base.indices[u[0]], self.base.indices[u[1]]
            Delta2_u = (u1 == u2) + 1.
            for j, u_p in enumerate(self.fields):
                u1_p, u2_p = self.base.indices[u_p[0]], self.base.indices[u_p[1]]
                Delta2_u_p = (u1_p == u2_p) + 1.
                inv_cov_sq = icov[u2_p, u1] * icov[u2, u1_p]
                inv_cov_sq += icov[u2_p, u2] * icov[u1, u1_p]
                fish_diag = 1. / (Delta2_u * Delta2_u_p) * np.sum(
                    self.base.m_weight * inv_cov_sq * self.all_ell_bins * self.beam_lm[u1] * self.beam_lm[u2]
                    * self.beam_lm[u1_p] * self.beam_lm[u2_p], axis=1)
                fish[i * self.Nl:(i + 1) * self.Nl, j * self.Nl:(j + 1) * self.Nl] = np.diag(np.real(fish_diag))
        self.fish_ideal = fish
        self.inv_fish_ideal = np.linalg.inv(self.fish_ideal)
        return fish

    def Cl_ideal(self, data, fish_ideal=[]):
        """Ideal estimator with analytic normalisation (polyspec/pspec_bin.py:262-287)."""
        if len(fish_ideal) != 0:
            self.fish_ideal = fish_ideal
            self.inv_fish_ideal = np.linalg.inv(fish_ideal)
        if not hasattr(self, 'inv_fish_ideal'):
            print("Computing ideal Fisher matrix")
            self.compute_fisher_ideal()
        Cl_num_ideal = np.concatenate(np.asarray(self.Cl_numerator_ideal(np.asarray(data) if not isinstance(data, torch.Tensor) else data.cpu().numpy())))
        Cl_out = np.matmul(self.inv_fish_ideal, Cl_num_ideal)
        Cl_dict = {}
        index = 0
        for u in self.fields:
            Cl_dict['%s' % u] = Cl_out[index:index + self.Nl]
            index += self.Nl
        return Cl_dict
