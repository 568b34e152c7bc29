"""ORACLE shim of the two ducc0 entry points the reference uses
(polyspec/base.py:70-74, 147-282), backed by the FP64 restatement in
oracle/sht_oracle.cpp.  Test infrastructure only."""
import numpy as np

from oracle import sht as _sht


def _nside(nphi):
    R = len(nphi)
    return (R + 1) // 4


class healpix:
    class Healpix_Base:
        def __init__(self, nside, scheme):
            assert scheme == "RING"
            self.nside = int(nside)

        def sht_info(self):
            g = _sht.ring_info(self.nside)
            return dict(theta=g["theta"], nphi=g["nphi"], phi0=g["phi0"], ringstart=g["ringstart"])


class sht:
    @staticmethod
    def synthesis(alm=None, lmax=None, spin=0, nthreads=0, mmax=None, theta_interpol=False, theta=None, nphi=None,
                  phi0=None, ringstart=None, **kw):
        assert mmax in (None, lmax)
        return _sht.synthesis(np.asarray(alm), lmax, spin, _nside(nphi), nthreads=nthreads)

    @staticmethod
    def adjoint_synthesis(lmax=None, spin=0, map=None, nthreads=0, mmax=None, theta_interpol=False, theta=None,
                          nphi=None, phi0=None, ringstart=None, **kw):
        assert mmax in (None, lmax)
        return _sht.adjoint_synthesis(np.asarray(map), lmax, spin, _nside(nphi), nthreads=nthreads)
