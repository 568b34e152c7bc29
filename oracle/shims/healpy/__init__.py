"""ORACLE shim of the healpy functions the reference's PSpecBin/Weightings path
uses (Alm.getlm, nside2npix, synalm).  Test infrastructure only.

``synalm`` is a documented generator of our own (healpy's internal draw order
is not reproducible here): one ``np.random.standard_normal((nfield, nalm, 2))``
call; m > 0 coefficients take (re + i im)/sqrt(2), m = 0 the first number; the
field correlation is applied with the symmetric square root of C_l.
"""
import numpy as np


class Alm:
    @staticmethod
    def getlm(lmax, i=None):
        m = np.concatenate([np.full(lmax + 1 - mm, mm, dtype=np.int64) for mm in range(lmax + 1)])
        l = np.concatenate([np.arange(mm, lmax + 1, dtype=np.int64) for mm in range(lmax + 1)])
        return l, m


def nside2npix(nside):
    return 12 * nside * nside


def synalm(cls, lmax=None, mmax=None, new=False, verbose=True):
    assert not new, "only the row ordering (new=False) is used by the reference"
    cls = [np.asarray(c) for c in cls]
    nfield = {1: 1, 6: 3}[len(cls)]
    l, m = Alm.getlm(lmax)
    z = np.random.standard_normal((nfield, len(l), 2))
    zc = np.where(m[None] > 0, (z[..., 0] + 1j * z[..., 1]) / np.sqrt(2.0), z[..., 0] + 0j)
    C = np.zeros((lmax + 1, nfield, nfield))
    k = 0
    for i in range(nfield):
        for j in range(i, nfield):
            C[:, i, j] = C[:, j, i] = cls[k][:lmax + 1]
            k += 1
    w, V = np.linalg.eigh(C)
    S = np.einsum("lij,lj,lkj->lik", V, np.sqrt(np.clip(w, 0.0, None)), V)
    return np.einsum("nij,jn->in", S[l], zc)


def get_all_neighbours(nside, theta, phi=None, nest=False, lonlat=False):
    raise NotImplementedError("inpainting is outside the oracle's scope")
