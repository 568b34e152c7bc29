"""ORACLE -- test infrastructure only (tests/, __graft_entry__.smoke(), the CPU
baseline of bench.py).  Never imported by the product package.

numpy restatement of the reference's S^-1 / PSpecBin path on top of the FP64
oracle SHT (oracle/sht_oracle.cpp), for use where the reference checkout is
absent (the GPU hosts).  It is pinned against the golden fixtures that the
unmodified reference produced (tests/golden/make_golden.py) by
tests/test_oracle_port.py.

Restated pieces and their reference lines:
  PortBase.to_lm / to_map          polyspec/base.py:131-176  (ducc0 calls -> oracle SHT)
  PortBase.applyAinv               polyspec/base.py:424-446
  PortBase.generate_data           polyspec/base.py:305-343  (add_B=False path; shim synalm)
  PortWeightings.__init__          polyspec/weighting.py:6-85
  PortWeightings.applySinv_ideal   polyspec/weighting.py:186-214
  PortWeightings.applySinv_optimal polyspec/weighting.py:148-184
  PortCGD                          polyspec/weighting.py:217-367
  PortPSpecBin                     polyspec/pspec_bin.py:20-164
"""
import numpy as np

from . import sht


def _getlm(lmax):
    return sht.getlm(lmax)


class PortBase:
    def __init__(self, Nside, Cl_tot, beam, pol=True, lmax=None, nthreads=0):
        self.Nside = Nside
        self.pol = pol
        self.Npix = 12 * Nside ** 2
        self.A_pix = 4 * np.pi / self.Npix
        self.lmax = 3 * Nside - 1 if lmax is None else int(lmax)
        self.l_arr, self.m_arr = _getlm(self.lmax)
        self.nthreads = nthreads or sht.default_threads()
        self.indices = {'T': 0, 'E': 1, 'B': 2}
        nf = 1 + 2 * pol
        L = self.lmax + 1
        self.Cl_tot = Cl_tot
        self.beam = np.asarray(beam)[:nf, :L]
        self.m_weight = 1. + 1. * (self.m_arr > 0)
        if pol:
            C = np.asarray([[Cl_tot['TT'], Cl_tot['TE'], Cl_tot['TB']], [Cl_tot['TE'], Cl_tot['EE'], Cl_tot['EB']],
                            [Cl_tot['TB'], Cl_tot['EB'], Cl_tot['BB']]])[:, :, :L]
            Cl = np.moveaxis(C, 2, 0)
            good = np.linalg.det(Cl) > 0
            inv = np.zeros((3, 3, L))
            inv[:, :, good] = np.moveaxis(np.linalg.inv(Cl[good]), 0, 2)
        else:
            tt = np.asarray(Cl_tot['TT'])[:L]
            inv = np.zeros((1, 1, L))
            inv[0, 0, tt > 0] = 1. / tt[tt > 0]
        self.inv_Cl_tot_mat = inv
        self.inv_Cl_tot_lm_mat = inv[:, :, self.l_arr]
        self.beam_lm = self.beam[:, self.l_arr]
        self.n_synth = 0
        self.n_adjoint = 0

    def to_lm(self, m, lmax=None):
        lmax = self.lmax if lmax is None else lmax
        m = np.asarray(m)
        scale = np.pi / (3. * self.Nside ** 2)
        self.n_adjoint += 1
        if len(m) == 3:
            T = sht.adjoint_synthesis(m[None, :1], lmax, 0, self.Nside, nthreads=self.nthreads)[0]
            EB = sht.adjoint_synthesis(m[None, 1:], lmax, 2, self.Nside, nthreads=self.nthreads)[0]
            return np.concatenate([T, EB]) * scale
        return sht.adjoint_synthesis(m.reshape(1, 1, -1), lmax, 0, self.Nside, nthreads=self.nthreads)[0] * scale

    def to_map(self, a, lmax=None):
        lmax = self.lmax if lmax is None else lmax
        a = np.asarray(a)
        self.n_synth += 1
        if len(a) == 3:
            T = sht.synthesis(a[None, :1], lmax, 0, self.Nside, nthreads=self.nthreads)[0]
            QU = sht.synthesis(a[None, 1:], lmax, 2, self.Nside, nthreads=self.nthreads)[0]
            return np.concatenate([T, QU])
        return sht.synthesis(a.reshape(1, 1, -1), lmax, 0, self.Nside, nthreads=self.nthreads)[0]

    def applyAinv(self, a, lmax=None):
        lmax = self.lmax if lmax is None else lmax
        f = self.l_arr <= lmax
        return self.beam_lm[:, f] * np.einsum('ijk,jk->ik', self.inv_Cl_tot_lm_mat[:, :, f], self.beam_lm[:, f] * a)

    def generate_data(self, seed, deconvolve_beam=True):
        """GRF alm from numpy's global generator (the documented synalm of oracle/shims/healpy)."""
        np.random.seed(seed)
        nf = 1 + 2 * self.pol
        rows = ([self.Cl_tot[k] for k in ('TT', 'TE', 'TB', 'EE', 'EB', 'BB')] if self.pol else [self.Cl_tot['TT']])
        l, m = self.l_arr, self.m_arr
        z = np.random.standard_normal((nf, len(l), 2))
        zc = np.where(m[None] > 0, (z[..., 0] + 1j * z[..., 1]) / np.sqrt(2.0), z[..., 0] + 0j)
        C = np.zeros((self.lmax + 1, nf, nf))
        k = 0
        for i in range(nf):
            for j in range(i, nf):
                C[:, i, j] = C[:, j, i] = np.asarray(rows[k])[:self.lmax + 1]
                k += 1
        w, V = np.linalg.eigh(C)
        S = np.einsum("lij,lj,lkj->lik", V, np.sqrt(np.clip(w, 0.0, None)), V)
        a = np.einsum("nij,jn->in", S[l], zc)
        if deconvolve_beam:
            b = self.beam_lm
            a = np.where(b != 0, a / np.where(b != 0, b, 1.0), 0.0)
        return a


class PortWeightings:
    def __init__(self, base, mask, Cl_raw, noise_cov):
        self.base = base
        self.mask = np.asarray(mask, dtype=np.float64).reshape(-1, base.Npix)
        self.pixel_area = 4 * np.pi / base.Npix
        nf = 1 + 2 * base.pol
        L = base.lmax + 1
        self.noise_cov = np.asarray(noise_cov, dtype=np.float64).reshape(nf, -1)
        self.noise_icov = np.zeros_like(self.noise_cov)
        nz = self.noise_cov != 0
        self.noise_icov[nz] = 1. / self.noise_cov[nz]
        self.Nl_iso = np.array([np.mean(self.noise_cov[i][self.mask[i] > 0.99]) * self.pixel_area for i in range(nf)])
        if base.pol:
            C = np.asarray([[Cl_raw['TT'], Cl_raw['TE'], Cl_raw['TB']], [Cl_raw['TE'], Cl_raw['EE'], Cl_raw['EB']],
                            [Cl_raw['TB'], Cl_raw['EB'], Cl_raw['BB']]])[:, :, :L]
            Cl = np.moveaxis(C, 2, 0)
            inv = np.zeros((3, 3, L))
            if np.sum(Cl_raw['BB']) == 0:
                good = np.linalg.det(Cl[:, :2, :2]) > 0
                inv[:2, :2, good] = np.moveaxis(np.linalg.inv(Cl[good, :2, :2]), 0, 2)
            else:
                good = np.linalg.det(Cl) > 0
                inv[:, :, good] = np.moveaxis(np.linalg.inv(Cl[good]), 0, 2)
        else:
            Cl = np.asarray(Cl_raw['TT'])[:L].reshape(-1, 1, 1)
            inv = np.zeros((1, 1, L))
            good = Cl[:, 0, 0] > 0
            inv[:, :, good] = np.moveaxis(np.linalg.inv(Cl[good]), 0, 2)
        self.Cl_l = Cl
        self.inv_Cl_lm = inv[:, :, base.l_arr]
        beam = base.beam
        invS = inv + np.einsum('il,jl,ij->ijl', beam, beam, np.diag(1. / self.Nl_iso))
        invS[:, :, :2] = invS[:, :, 2:3]
        self.Sigma_lm = np.moveaxis(np.linalg.inv(np.moveaxis(invS, 2, 0)), 0, 2)[:, :, base.l_arr]
        self.x0op_lm = np.einsum('lab,bl,bcl->acl', Cl, beam, base.inv_Cl_tot_mat)[:, :, base.l_arr]

    def applySinv_ideal(self, m, lmax=None):
        lmax = self.base.lmax if lmax is None else lmax
        f = self.base.l_arr <= lmax
        a = self.base.to_lm(m)
        return self.base.beam_lm[:, f] * np.einsum("abl,bl->al", self.base.inv_Cl_tot_lm_mat[:, :, f], a[:, f])

    def applySinv_optimal(self, d, preconditioner='harmonic', nstep=25, thresh=1e-4, lmax=None):
        lmax = self.base.lmax if lmax is None else lmax
        x0 = np.einsum('abi,bi->ai', self.x0op_lm, self.base.to_lm(d))
        cg = PortCGD(self, d, x0, preconditioner)
        cg.run(nstep, thresh)
        self.last_cgd = cg
        return cg.get_ivar_lm()[:, self.base.l_arr <= lmax]


class PortCGD:
    def __init__(self, W, d, x0, preconditioner='harmonic', test_b=None):
        self.W = W
        self.base = W.base
        self.preconditioner = preconditioner
        b0 = self._get_b(d) if test_b is None else test_b.copy()
        self.x0 = x0 if x0 is not None else 0.
        b = b0 - self._apply_A(x0) if x0 is not None else b0
        self.x = np.zeros_like(b)
        self.r = b.copy()
        z = self._apply_M(self.r)
        self.rz = self.dot(self.r, z)
        self.rz0 = float(self.dot(b0, self._apply_M(b0)))
        self.p = z
        self.i = 0
        self.err = self.rz / self.rz0

    def dot(self, a, b):
        return np.sum(a * np.conj(b) * self.base.m_weight).real

    def _get_b(self, d):
        return self.base.beam_lm * self.base.to_lm(self.W.mask * (d * self.W.noise_icov / self.W.pixel_area))

    def _apply_Cinv(self, a):
        return np.einsum('abi,bi->ai', self.W.inv_Cl_lm, a)

    def _apply_A(self, a):
        m = self.W.mask * self.base.to_map(a * self.base.beam_lm)
        m = self.W.mask * (m * self.W.noise_icov / self.W.pixel_area)
        return self._apply_Cinv(a) + self.base.beam_lm * self.base.to_lm(m)

    def _apply_M(self, a):
        if self.preconditioner == 'harmonic':
            return np.einsum('abi,bi->ai', self.W.Sigma_lm, a)
        alm = np.einsum('abi,bi->ai', self.W.Sigma_lm, a)
        sig = self._apply_Cinv(alm)
        noi = alm * self.base.beam_lm / self.W.Nl_iso[:, None]
        noi = self.base.to_lm(self.W.noise_cov * self.base.to_map(noi)) * self.W.pixel_area
        noi *= self.base.beam_lm / self.W.Nl_iso[:, None]
        return np.einsum('abi,bi->ai', self.W.Sigma_lm, noi + sig)

    def step(self):
        Ap = self._apply_A(self.p)
        alpha = self.rz / self.dot(self.p, Ap)
        self.x += alpha * self.p
        self.r -= alpha * Ap
        z = self._apply_M(self.r)
        nrz = self.dot(self.r, z)
        self.err = nrz / self.rz0
        beta = nrz / self.rz
        self.rz = nrz
        self.p = z + beta * self.p
        self.i += 1

    def run(self, nstep, thresh):
        for _ in range(nstep):
            self.step()
            if self.err < thresh:
                break

    def get_ivar_lm(self):
        return self._apply_Cinv(self.x + self.x0)


class PortPSpecBin:
    def __init__(self, base, mask, applySinv, l_bins, fields):
        self.base = base
        self.mask = np.asarray(mask, dtype=np.float64)
        self.applySinv = applySinv
        self.l_bins = np.asarray(l_bins)
        self.Nl = len(l_bins) - 1
        self.fields = list(fields)
        self.N_p = len(self.fields) * self.Nl
        self.ell_bins = [(base.l_arr >= l_bins[b]) & (base.l_arr < l_bins[b + 1]) for b in range(self.Nl)]
        self.all_ell_bins = np.vstack(self.ell_bins)

    def Cl_numerator(self, data):
        h = self.applySinv(data)
        out = []
        for u in self.fields:
            u1, u2 = self.base.indices[u[0]], self.base.indices[u[1]]
            out.append(np.real(1. / ((u1 == u2) + 1.) * np.sum(self.base.m_weight * np.conj(h[u1]) * h[u2]
                                                                 * self.all_ell_bins, axis=1)))
        return np.asarray(out)

    def compute_fisher_contribution(self, seed=None, a_lm=None):
        if a_lm is None:
            a_lm = self.base.generate_data(seed + int(1e7), deconvolve_beam=True)
        bl = self.base.beam_lm

        def rows(U):
            out = []
            for u in self.fields:
                u1, u2 = self.base.indices[u[0]], self.base.indices[u[1]]
                V = np.zeros_like(U)
                V[u1] += U[u2]
                V[u2] += U[u1]
                for b in range(self.Nl):
                    out.append(V * self.ell_bins[b] / ((u1 == u2) + 1.))
            return out

        US = self.applySinv(self.mask * self.base.to_map(bl * a_lm))
        QS = np.asarray([(self.base.m_weight * r).ravel() for r in rows(US)])
        UA = self.base.applyAinv(a_lm)
        QA = np.asarray([self.applySinv(self.mask * self.base.to_map(bl * r)).ravel() for r in rows(UA)])
        return 0.5 * np.real(QS.conj() @ QA.T)
