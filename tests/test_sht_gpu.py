"""FP64 CUDA SHT against the FP64 oracle (restated HEALPix/ducc0 transforms).

Tolerance: the plain FP64 backend must agree with the oracle to 1e-10
relative error in max-norm (maps and alm).
"""
import numpy as np
import pytest

from oracle import sht as osht

TOL = 1e-10


def rand_alm(rng, lmax, lead=()):
    n = osht.nalm(lmax)
    a = rng.normal(size=lead + (n,)) + 1j * rng.normal(size=lead + (n,))
    l, m = osht.getlm(lmax)
    a[..., m == 0] = a[..., m == 0].real
    return a


def relerr(x, ref):
    return np.abs(x - ref).max() / max(np.abs(ref).max(), 1e-300)


@pytest.mark.gpu
@pytest.mark.parametrize("nside,lfac", [(2, 3), (4, 3), (8, 3), (16, 2), (16, 3), (32, 3), (64, 2)])
@pytest.mark.parametrize("spin", [0, 1, 2, 3])
@pytest.mark.parametrize("batch", [1, 3])
def test_synthesis_adjoint_vs_oracle(nside, lfac, spin, batch):
    import torch
    from polyspec_b200.sht import SHTPlan
    lmax = lfac * nside - 1 if lfac == 3 else lfac * nside
    rng = np.random.default_rng(1000 * nside + 10 * spin + batch)
    ncomp = 1 if spin == 0 else 2
    alm = rand_alm(rng, lmax, (batch, ncomp))
    l, m = osht.getlm(lmax)
    alm[..., l < spin] = 0
    ref_map = osht.synthesis(alm, lmax, spin, nside)
    plan = SHTPlan(nside, lmax)
    a_t = torch.from_numpy(alm if spin > 0 else alm[:, 0]).cuda()
    out = plan.synthesis(a_t, spin).cpu().numpy()
    if spin == 0:
        out = out[:, None]
    assert relerr(out, ref_map) < TOL
    mp = rng.normal(size=(batch, ncomp, 12 * nside * nside))
    ref_alm = osht.adjoint_synthesis(mp, lmax, spin, nside) * 0.5
    m_t = torch.from_numpy(mp if spin > 0 else mp[:, 0]).cuda()
    out_alm = plan.adjoint(m_t, spin, scale=0.5).cpu().numpy()
    if spin == 0:
        out_alm = out_alm[:, None]
    assert relerr(out_alm, ref_alm) < TOL
