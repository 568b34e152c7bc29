"""ORACLE -- test infrastructure only (tests/, __graft_entry__.smoke(), bench.py's
CPU-baseline leg).  Never imported by the product package.

ctypes front end of ``liborc_sht.so`` (``sht_oracle.cpp``): an FP64 CPU
restatement of the two ducc0 calls the reference makes for its SHTs,

* ``ducc0.sht.synthesis``          (polyspec/base.py:172-176, 225, 230-231, 282)
* ``ducc0.sht.adjoint_synthesis``  (polyspec/base.py:147-151, 193, 206, 253)

with ducc0's array conventions: ``alm[..., ncomp, nalm]`` complex128 in the
m-major HEALPix order ``idx = m(2 lmax + 1 - m)/2 + l``, maps
``[..., ncomp, npix]`` float64 in RING order, ``ncomp = 1`` for spin 0 and
``2`` (G, C <-> Q, U) for spin > 0.  ``adjoint_synthesis`` carries no
quadrature weight: the reference multiplies by ``pi/(3 nside^2)`` itself.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liborc_sht.so")
        if not os.path.exists(path):
            import subprocess
            subprocess.check_call(["make", "-s", "-C", _HERE])
        L = ctypes.CDLL(path)
        i, d, p = ctypes.c_int, ctypes.c_double, ctypes.c_void_p
        L.orc_ring_info.argtypes = [i, p, p, p, p]
        L.orc_legendre.argtypes = [i, i, i, i, i, p, p]
        L.orc_synthesis.argtypes = [i, i, i, i, i, p, p, i, i]
        L.orc_adjoint.argtypes = [i, i, i, i, i, p, p, i, i]
        for f in (L.orc_ring_info, L.orc_legendre, L.orc_synthesis, L.orc_adjoint):
            f.restype = i
        _LIB = L
    return _LIB


def default_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:  # pragma: no cover
        return os.cpu_count() or 1


def nalm(lmax):
    return (lmax + 1) * (lmax + 2) // 2


def getlm(lmax):
    """(l, m) of every alm in the m-major order (healpy.Alm.getlm, used at polyspec/base.py:31)."""
    m = np.concatenate([np.full(lmax + 1 - mm, mm) for mm in range(lmax + 1)])
    l = np.concatenate([np.arange(mm, lmax + 1) for mm in range(lmax + 1)])
    return l, m


def ring_info(nside):
    """theta, phi0, nphi, ringstart of the HEALPix RING scheme (ducc0 Healpix_Base.sht_info())."""
    R = 4 * nside - 1
    theta = np.zeros(R)
    phi0 = np.zeros(R)
    nphi = np.zeros(R, dtype=np.int64)
    rs = np.zeros(R, dtype=np.int64)
    rc = lib().orc_ring_info(nside, theta.ctypes.data, phi0.ctypes.data, nphi.ctypes.data, rs.ctypes.data)
    assert rc == 0
    return dict(theta=theta, phi0=phi0, nphi=nphi, ringstart=rs)


def legendre(nside, ring, lmax, m, spin=0):
    """lam_lm(theta_ring) for l = m..lmax (spin 0), or (F+, F-) for spin > 0."""
    a = np.zeros(lmax - m + 1)
    b = np.zeros(lmax - m + 1)
    rc = lib().orc_legendre(nside, ring, lmax, m, spin, a.ctypes.data, b.ctypes.data)
    assert rc == 0
    return a if spin == 0 else (a, b)


def _nside_from_geom(nphi):
    R = len(nphi)
    nside = (R + 1) // 4
    assert 4 * nside - 1 == R, "only full HEALPix RING geometries are supported"
    return nside


def synthesis(alm, lmax, spin, nside, mmax=None, nthreads=0, direct=False):
    """alm[..., ncomp, nalm] -> map[..., ncomp, npix]."""
    mmax = lmax if mmax is None else mmax
    alm = np.ascontiguousarray(alm, dtype=np.complex128)
    ncomp = 1 if spin == 0 else 2
    assert alm.shape[-2] == ncomp and alm.shape[-1] == nalm(lmax), alm.shape
    lead = alm.shape[:-2]
    nmaps = int(np.prod(lead)) if lead else 1
    out = np.zeros(lead + (ncomp, 12 * nside * nside))
    rc = lib().orc_synthesis(nside, lmax, mmax, spin, nmaps, alm.ctypes.data, out.ctypes.data,
                             nthreads or default_threads(), int(direct))
    if rc != 0:
        raise ValueError("orc_synthesis failed (%d)" % rc)
    return out


def adjoint_synthesis(map, lmax, spin, nside, mmax=None, nthreads=0, direct=False):
    """map[..., ncomp, npix] -> alm[..., ncomp, nalm] (no quadrature weights)."""
    mmax = lmax if mmax is None else mmax
    map = np.ascontiguousarray(map, dtype=np.float64)
    ncomp = 1 if spin == 0 else 2
    assert map.shape[-2] == ncomp and map.shape[-1] == 12 * nside * nside, map.shape
    lead = map.shape[:-2]
    nmaps = int(np.prod(lead)) if lead else 1
    out = np.zeros(lead + (ncomp, nalm(lmax)), dtype=np.complex128)
    rc = lib().orc_adjoint(nside, lmax, mmax, spin, nmaps, map.ctypes.data, out.ctypes.data,
                           nthreads or default_threads(), int(direct))
    if rc != 0:
        raise ValueError("orc_adjoint failed (%d)" % rc)
    return out
