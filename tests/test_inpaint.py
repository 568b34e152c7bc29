"""Inpainting (Weightings.inpaint_map, polyspec/weighting.py:87-146) and the HEALPix
neighbour table it runs on.

CPU: the oracle's neighbour relation (oracle/healpix_nb.py, derived from shared
pixel vertices since healpy is absent) is symmetric, has 8 distinct neighbours per
pixel except 24 slots of -1 (where three faces meet), and its inpainting fills
every hole.  GPU: ps_healpix_neighbours equals the oracle's table exactly for
Nside 1-32, and inpaint_map (fill passes + 50 smoothing passes) equals the oracle's
restatement of the reference bit for bit (the same neighbour order, sums in the
same order), for T and T, Q, U maps, masked and unmasked inputs.
"""
import numpy as np
import pytest

NSIDES = (1, 2, 3, 4, 8, 16, 32)


def _holes(nside, nb, seed, layers=2, ncentres=6):
    rng = np.random.default_rng(seed)
    sel = set(int(p) for p in rng.choice(12 * nside * nside, ncentres, replace=False))
    for _ in range(layers):
        sel |= set(int(q) for p in list(sel) for q in nb[p] if q >= 0)
    m = np.zeros(12 * nside * nside)
    m[list(sel)] = 1.
    return m


@pytest.mark.parametrize("nside", (1, 2, 4, 8))
def test_oracle_neighbours(nside):
    from oracle.healpix_nb import all_neighbours, xyf2ring
    nb = all_neighbours(nside)
    npix = 12 * nside * nside
    f, y, x = np.meshgrid(np.arange(12), np.arange(nside), np.arange(nside), indexing='ij')
    assert np.array_equal(np.sort(xyf2ring(nside, f.ravel(), x.ravel(), y.ravel())), np.arange(npix))
    assert (nb < 0).sum() == 24
    for p in range(npix):
        row = nb[p][nb[p] >= 0]
        assert len(set(row)) == len(row) and p not in row
        for q in row:
            assert p in nb[q]


def test_oracle_inpaint_fills_holes():
    from oracle.healpix_nb import all_neighbours, inpaint_map
    nside = 8
    nb = all_neighbours(nside)
    mask = _holes(nside, nb, 1)
    rng = np.random.default_rng(2)
    m = (1. + rng.normal(size=(1, 12 * nside * nside))) * (1. - mask)[None]
    out = inpaint_map(m, mask[None], nside, False, neighbours=nb)
    assert np.all(out[0][mask == 1] != 0)
    assert np.array_equal(out[0][mask == 0], m[0][mask == 0])


@pytest.mark.gpu
@pytest.mark.parametrize("nside", NSIDES)
def test_neighbour_table(nside):
    import torch
    from oracle.healpix_nb import all_neighbours
    from polyspec_b200 import healpix
    nb = healpix.neighbours(nside, torch.device("cuda")).cpu().numpy()
    assert np.array_equal(nb, all_neighbours(nside))


@pytest.mark.gpu
@pytest.mark.parametrize("pol", [False, True])
@pytest.mark.parametrize("masked", [True, False])
def test_inpaint_map(pol, masked):
    import torch
    from oracle.healpix_nb import all_neighbours, inpaint_map
    from polyspec_b200 import PolySpec, Weightings
    from polyspec_b200.workloads import fiducial_cl, total_cl, gaussian_beam, noise_cl
    nside = 32
    nb = all_neighbours(nside)
    nf = 3 if pol else 1
    imask = np.stack([_holes(nside, nb, 10 + i) for i in range(nf)])
    lmax = 3 * nside - 1
    cl = fiducial_cl(lmax, pol)
    beam = np.stack([gaussian_beam(lmax, 30.)] * nf)
    cltot = total_cl(cl, beam, noise_cl(nside, lmax, 30.0, pol))
    base = PolySpec(nside, dict(cltot), beam=list(beam), pol=pol, backend="cuda")
    wts = Weightings(base, np.ones((nf, 12 * nside * nside)), dict(cl), inpainting_mask=imask)
    rng = np.random.default_rng(3)
    m = 1. + rng.normal(size=(nf, 12 * nside * nside))
    if masked:
        m = m * (1. - imask)
    got = wts.inpaint_map(m)
    ref = inpaint_map(m, imask, nside, pol, neighbours=nb)
    assert np.array_equal(got, ref)
    # the ideal filter inpaints first
    a = wts.applySinv_ideal(m)
    wts2 = Weightings(base, np.ones((nf, 12 * nside * nside)), dict(cl))
    b = wts2.applySinv_ideal(ref)
    assert np.abs(a - b).max() <= 1e-14 * np.abs(b).max()
