"""The FP64 oracle pinned by identities and closed forms (the reference has
no golden vectors for the SHT: ducc0 is third-party and absent here)."""
from math import comb, factorial, pi, sqrt

import numpy as np
import pytest

from oracle import sht


def goldberg(s, l, m, th):
    """sY_lm(theta, 0), Goldberg et al. (1967) explicit sum."""
    if l < max(abs(m), abs(s)):
        return np.zeros_like(th)
    pref = (-1) ** abs(m) * sqrt((2 * l + 1) / (4 * pi) * factorial(l + m) * factorial(l - m)
                                 / (factorial(l + s) * factorial(l - s)))
    tot = np.zeros_like(th)
    for r in range(0, l - s + 1):
        k = r + s - m
        if k < 0 or k > l + s:
            continue
        tot = tot + comb(l - s, r) * comb(l + s, k) * (-1) ** (l - r - s) * (1 / np.tan(th / 2)) ** (2 * r + s - m)
    return pref * np.sin(th / 2) ** (2 * l) * tot


def pix_angles(nside):
    g = sht.ring_info(nside)
    th = np.concatenate([np.full(n, t) for t, n in zip(g['theta'], g['nphi'])])
    ph = np.concatenate([p0 + 2 * np.pi * np.arange(n) / n for p0, n in zip(g['phi0'], g['nphi'])])
    return th, ph


def rand_alm(rng, lmax, lead=()):
    l, m = sht.getlm(lmax)
    a = rng.normal(size=lead + (len(l),)) + 1j * rng.normal(size=lead + (len(l),))
    a[..., m == 0] = a[..., m == 0].real
    return a


def test_ring_geometry():
    for nside in (1, 2, 8, 32):
        g = sht.ring_info(nside)
        assert g['nphi'].sum() == 12 * nside ** 2
        assert np.all(np.diff(g['ringstart']) == g['nphi'][:-1])
        assert np.all(np.diff(g['theta']) > 0)
        # equal-area pixels: ring areas follow 2 pi (z_{i-1/2} - z_{i+1/2})
        assert abs(g['theta'][2 * nside - 1] - np.pi / 2) < 1e-15


@pytest.mark.parametrize("spin", [0, 1, 2, 3])
def test_synthesis_matches_goldberg(spin):
    nside, lmax = 8, 12
    th, ph = pix_angles(nside)
    l, m = sht.getlm(lmax)
    rng = np.random.default_rng(spin)
    if spin == 0:
        a = rand_alm(rng, lmax)
        ref = np.zeros(len(th))
        for i, (ll, mm) in enumerate(zip(l, m)):
            ref += (a[i] * goldberg(0, ll, mm, th) * np.exp(1j * mm * ph)).real * (1 if mm == 0 else 2)
        out = sht.synthesis(a[None, None], lmax, 0, nside)[0, 0]
        assert np.abs(out - ref).max() < 1e-12 * np.abs(ref).max()
        return
    G, C = rand_alm(rng, lmax, (2,))
    G[l < spin] = 0
    C[l < spin] = 0
    P = np.zeros(len(th), complex)
    for i, (ll, mm) in enumerate(zip(l, m)):
        P += -(G[i] + 1j * C[i]) * goldberg(spin, ll, mm, th) * np.exp(1j * mm * ph)
        if mm > 0:
            san = -((-1) ** mm) * (np.conj(G[i]) + 1j * np.conj(C[i]))
            P += san * goldberg(spin, ll, -mm, th) * np.exp(-1j * mm * ph)
    out = sht.synthesis(np.array([G, C])[None], lmax, spin, nside)[0]
    scale = np.abs(P).max()
    assert np.abs(out[0] - P.real).max() < 1e-12 * scale
    assert np.abs(out[1] - P.imag).max() < 1e-12 * scale


@pytest.mark.parametrize("spin", [0, 1, 2, 3])
def test_adjointness_and_dft_modes(spin):
    nside, lmax = 8, 23
    rng = np.random.default_rng(10 + spin)
    nc = 1 if spin == 0 else 2
    a = rand_alm(rng, lmax, (1, nc))
    mp = rng.normal(size=(1, nc, 12 * nside ** 2))
    Ya = sht.synthesis(a, lmax, spin, nside)
    Ytm = sht.adjoint_synthesis(mp, lmax, spin, nside)
    _, m = sht.getlm(lmax)
    lhs = np.sum(Ya * mp)
    rhs = np.sum((1 + (m > 0)) * (np.conj(a) * Ytm).real)
    assert abs(lhs - rhs) < 1e-12 * abs(lhs)
    assert np.abs(sht.synthesis(a, lmax, spin, nside, direct=True) - Ya).max() < 1e-12 * np.abs(Ya).max()
    assert np.abs(sht.adjoint_synthesis(mp, lmax, spin, nside, direct=True) - Ytm).max() < 1e-12 * np.abs(Ytm).max()


def test_spin1_gradient_convention():
    """HEALPix convention: the spin-1 transform of G = sqrt(l(l+1)) a_lm, C = 0 is the
    gradient (d_theta f, d_phi f / sin theta) of the scalar field f."""
    nside, lmax = 8, 10
    th, ph = pix_angles(nside)
    l, m = sht.getlm(lmax)
    a = rand_alm(np.random.default_rng(3), lmax)
    h = 1e-6

    def field(tt, pp):
        out = np.zeros(len(tt))
        for i, (ll, mm) in enumerate(zip(l, m)):
            out += (a[i] * goldberg(0, ll, mm, tt) * np.exp(1j * mm * pp)).real * (1 if mm == 0 else 2)
        return out
    dth = (field(th + h, ph) - field(th - h, ph)) / (2 * h)
    dph = (field(th, ph + h) - field(th, ph - h)) / (2 * h) / np.sin(th)
    G = np.sqrt(l * (l + 1.0)) * a
    out = sht.synthesis(np.array([G, 0 * G])[None], lmax, 1, nside)[0]
    assert np.abs(out[0] - dth).max() < 1e-7 * np.abs(dth).max()
    assert np.abs(out[1] - dph).max() < 1e-7 * np.abs(dph).max()


def test_high_order_seeds_are_finite():
    """Scaled seeds: high m near the pole underflows FP64 without rescaling."""
    nside, lmax = 256, 767
    lam = sht.legendre(nside, 0, lmax, 700, 0)
    assert np.all(np.isfinite(lam))
    lam2 = sht.legendre(nside, 511, lmax, 700, 0)
    assert np.all(np.isfinite(lam2)) and np.abs(lam2).max() > 1e-3
    fp, fm = sht.legendre(nside, 3, lmax, 600, 2)
    assert np.all(np.isfinite(fp)) and np.all(np.isfinite(fm))
