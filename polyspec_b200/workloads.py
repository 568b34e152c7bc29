"""Seeded synthetic inputs of the benchmark workloads (no datasets are used).

Stand-ins for the Planck-like inputs of the reference's scripts
(run_planck_local_trispectra.py, run_planck_binned_bispectrum.py):

* fiducial spectra  C_l^TT = 1000/(l+10)^2 uK^2, C^EE = 0.05 C^TT,
  C^TE = 0.3 sqrt(C^TT C^EE), C^BB = 1e-6 C^EE, C^TB = C^EB = 0;
* Gaussian beams  b_l = exp(-l(l+1) sigma^2/2), sigma = FWHM/sqrt(8 ln 2);
* masks: a Galactic-latitude cut with a cosine taper, and a boolean sky cut
  plus circular point-source holes at seeded uniform positions;
* white noise of a given depth (uK arcmin) per pixel, twice the variance in Q, U.

Pixel positions come from the HEALPix RING formulas (Gorski et al. 2005).
"""
import numpy as np


def fiducial_cl(lmax, pol=True, amp=1000.0):
    l = np.arange(lmax + 1, dtype=np.float64)
    tt = amp / (l + 10.0) ** 2
    if not pol:
        return {'TT': tt}
    ee = 0.05 * tt
    te = 0.3 * np.sqrt(tt * ee)
    bb = 1e-6 * ee
    z = 0.0 * tt
    return {'TT': tt, 'TE': te, 'TB': z.copy(), 'EE': ee, 'EB': z.copy(), 'BB': bb}


def gaussian_beam(lmax, fwhm_arcmin):
    sigma = np.radians(fwhm_arcmin / 60.0) / np.sqrt(8.0 * np.log(2.0))
    l = np.arange(lmax + 1, dtype=np.float64)
    return np.exp(-l * (l + 1.0) * sigma ** 2 / 2.0)


def pixel_z_phi(nside):
    """cos(theta) and longitude of every RING pixel centre."""
    ns = nside
    npix = 12 * ns * ns
    z = np.empty(npix)
    phi = np.empty(npix)
    for i in range(1, 4 * ns):
        north = i <= 2 * ns
        ii = i if north else 4 * ns - i
        if ii < ns:
            t = ii * ii / (3.0 * ns * ns)
            zz = 1.0 - t if north else t - 1.0
            n = 4 * ii
            start = 2 * ii * (ii - 1) if north else npix - 2 * ii * (ii + 1)
            p = (np.arange(n) + 0.5) * (np.pi / (2.0 * ii))
        else:
            zz = (2 * ns - i) * 2.0 / (3.0 * ns)
            n = 4 * ns
            start = 2 * ns * (ns - 1) + (i - ns) * 4 * ns
            shift = 0.5 if (i - ns) % 2 == 0 else 0.0
            p = (np.arange(n) + shift) * (np.pi / (2.0 * ns))
        z[start:start + n] = zz
        phi[start:start + n] = p
    return z, phi


def latitude_mask(nside, cut_deg=15.0, taper_deg=5.0):
    """0 for |lat| < cut, 1 above cut + taper, 0.5 (1 - cos(pi (|lat|-cut)/taper)) between."""
    z, _ = pixel_z_phi(nside)
    lat = np.degrees(np.arcsin(np.clip(z, -1, 1)))
    a = np.abs(lat)
    m = np.where(a < cut_deg, 0.0, np.where(a > cut_deg + taper_deg, 1.0,
                                            0.5 * (1.0 - np.cos(np.pi * (a - cut_deg) / taper_deg))))
    return m


def point_source_mask(nside, cut_deg=5.74, n_holes=500, radius_arcmin=10.0, seed=0):
    """Boolean mask: |lat| < cut removed, plus n_holes discs at seeded uniform positions.

    RING order sorts pixels by decreasing z, so each disc only scans the pixel
    range of its z band."""
    z, phi = pixel_z_phi(nside)
    lat = np.degrees(np.arcsin(np.clip(z, -1, 1)))
    m = np.abs(lat) >= cut_deg
    rng = np.random.default_rng(seed)
    zc = rng.uniform(-1.0, 1.0, n_holes)
    pc = rng.uniform(0.0, 2 * np.pi, n_holes)
    rad = np.radians(radius_arcmin / 60.0)
    cr = np.cos(rad)
    negz = -z
    for k in range(n_holes):
        stc = np.sqrt(max(1 - zc[k] ** 2, 0.0))
        lo = np.searchsorted(negz, -(zc[k] + 1.5 * rad), side="left")
        hi = np.searchsorted(negz, -(zc[k] - 1.5 * rad), side="right")
        zz = z[lo:hi]
        st = np.sqrt(np.clip(1 - zz * zz, 0, None))
        cosd = zz * zc[k] + st * stc * np.cos(phi[lo:hi] - pc[k])
        m[lo:hi][cosd > cr] = False
    return m.astype(np.float64)


def white_noise_cov(nside, depth_uk_arcmin=30.0, pol=True):
    """Per-pixel noise variance (uK^2): depth^2 / Omega_pix (arcmin^2), x2 for Q and U."""
    omega = 4 * np.pi / (12 * nside * nside) * (180 * 60 / np.pi) ** 2
    s2 = depth_uk_arcmin ** 2 / omega
    npix = 12 * nside * nside
    if not pol:
        return np.full((1, npix), s2)
    return np.stack([np.full(npix, s2), np.full(npix, 2 * s2), np.full(npix, 2 * s2)])


def noise_cl(nside, lmax, depth_uk_arcmin=30.0, pol=True):
    """White-noise power N_l = depth^2 (in uK^2 sr) for T, x2 for E/B."""
    n = (depth_uk_arcmin * np.pi / (180 * 60)) ** 2
    out = {'TT': np.full(lmax + 1, n)}
    if pol:
        out.update({'EE': np.full(lmax + 1, 2 * n), 'BB': np.full(lmax + 1, 2 * n)})
    return out


def total_cl(cl, beam, nl=None):
    """C_tot = b^2 C + N (beam-convolved signal plus noise), as the reference's Cl_tot expects."""
    out = {}
    for k, v in cl.items():
        b1 = beam[{'T': 0, 'E': 1, 'B': 2}[k[0]]] if np.ndim(beam) == 2 else beam
        b2 = beam[{'T': 0, 'E': 1, 'B': 2}[k[1]]] if np.ndim(beam) == 2 else beam
        out[k] = b1 * b2 * v
        if nl is not None and k in nl:
            out[k] = out[k] + nl[k]
    return out


def cg_fisher_setup(nside=1024, lmax=2048, n_holes=500, depth=30.0, fwhm_arcmin=5.0, nbins=8, seed=0,
                    fields=('TT', 'TE', 'EE', 'BB')):
    """The masked-CG PSpecBin workload: TEB at (nside, lmax), white noise of
    `depth` uK arcmin, a |lat| < 5.74 deg cut (10% of the sky) plus `n_holes`
    point-source holes of 10' radius, `nbins` linear bins in [2, lmax].

    Returns (cl_raw, cl_tot, beam[3, lmax+1], mask[3, npix], noise_cov[3, npix], l_bins).
    """
    cl = fiducial_cl(lmax, True)
    b = gaussian_beam(lmax, fwhm_arcmin)
    beam = np.stack([b, b, b])
    nl = noise_cl(nside, lmax, depth, True)
    cltot = total_cl(cl, beam, nl)
    m = point_source_mask(nside, 5.74, n_holes, 10.0, seed)
    mask = np.stack([m, m, m])
    noise = white_noise_cov(nside, depth, True)
    l_bins = np.linspace(2, lmax, nbins + 1).astype(int)
    return cl, cltot, beam, mask, noise, l_bins


def anisotropic_noise_setup(nside, lmax, amp=3.0, depth=30.0, fwhm_arcmin=5.0, seed=0):
    """Full-sky TEB workload with latitude-dependent white noise: the pixel noise
    variance of the 30 uK' map is multiplied by 1 + amp z^2 (a deep equator, as a
    scan strategy that crosses the poles less often would give).  Returns
    (cl_raw, cl_tot, beam[3, lmax+1], mask[3, npix] (ones), noise_cov[3, npix])."""
    cl = fiducial_cl(lmax, True)
    b = gaussian_beam(lmax, fwhm_arcmin)
    beam = np.stack([b, b, b])
    nl = noise_cl(nside, lmax, depth, True)
    cltot = total_cl(cl, beam, nl)
    z, _ = pixel_z_phi(nside)
    noise = white_noise_cov(nside, depth, True) * (1.0 + amp * z * z)[None, :]
    mask = np.ones((3, 12 * nside * nside))
    return cl, cltot, beam, mask, noise


def bispec_setup(nside=256, lmax=511, nbins=10, fwhm_arcmin=30.0, pol=True):
    """Binned-bispectrum workload: T and E (TTT, TTE, TEE, EEE), nbins log-spaced
    l-bins in [2, lmax], fiducial spectra, Gaussian beam, the latitude mask
    (|b| < 15 deg, 5 deg cosine taper) and the ideal S^-1 filter.  Returns
    (Cl_tot, Cl_raw, beam rows, mask, l_bins, fields)."""
    cl = fiducial_cl(lmax, pol)
    b = gaussian_beam(lmax, fwhm_arcmin)
    nf = 3 if pol else 1
    beam = np.stack([b] * nf)
    nl = noise_cl(nside, lmax, 30.0, pol)
    cltot = total_cl(cl, beam, nl)
    mask = latitude_mask(nside, 15.0, 5.0)
    l_bins = np.unique(np.round(np.geomspace(2, lmax, nbins + 1)).astype(int))
    fields = ['TTT', 'TTE', 'TEE', 'EEE'] if pol else ['TTT']
    return cltot, cl, beam, mask, l_bins, fields


def smooth_transfer(npol, k_arr, lmax, seed=3):
    """Seeded smooth stand-in transfer functions T_l^X(k) [npol, lmax+1, nk]: sums of
    Gaussian bumps in (log k, l), zero at l = 0, 1."""
    rng = np.random.default_rng(seed)
    l = np.arange(lmax + 1)[:, None]
    lk = np.log(k_arr)[None, :]
    T = np.zeros((npol, lmax + 1, len(k_arr)))
    for X in range(npol):
        for _ in range(8):
            a = rng.normal() * (0.3 if X else 1.0)
            lc = rng.uniform(np.log(2e-4), np.log(0.08))
            sl = rng.uniform(0.4, 1.2)
            l0 = rng.uniform(0, lmax)
            s0 = rng.uniform(0.05, 0.3) * lmax
            T[X] += a * np.exp(-(lk - lc) ** 2 / (2 * sl ** 2) - (l - l0) ** 2 / (2 * s0 ** 2))
    T[:, :2] = 0.
    return T


def tspec_setup(nside=512, lmax=1000, n_r=24, nk=400, fwhm_arcmin=10.0, pol=True, seed=0, n_rtau=(4, 4)):
    """Template-trispectrum workload: seeded smooth transfer functions on nk log-spaced
    k in [1e-4, 0.1], n_r radial samples around recombination with seeded weights (the
    same weights for gNL-loc, gNL-con and tauNL-loc), an n_rtau[0] x n_rtau[1] grid of
    (r, tau) samples (r in [13400, 14200] Mpc, tau in [-2000, -50] Mpc) with seeded
    weights for the EFTI shapes, C_phi = 1e-7 / (L (L+1))^2, the fiducial spectra as
    lensing weights, Gaussian beam, latitude mask, ideal S^-1 filter.  Returns a dict
    of the TSpecTemplate arguments and the base's inputs."""
    base_lmax = 3 * nside - 1
    cl = fiducial_cl(base_lmax, pol)
    b = gaussian_beam(base_lmax, fwhm_arcmin)
    nf = 3 if pol else 1
    beam = np.stack([b] * nf)
    nl = noise_cl(nside, base_lmax, 30.0, pol)
    cltot = total_cl(cl, beam, nl)
    mask = latitude_mask(nside, 15.0, 5.0)
    k_arr = np.geomspace(1e-4, 0.1, nk)
    rng = np.random.default_rng(seed + 1)
    r_values = np.linspace(13300., 14400., n_r)
    weights = rng.uniform(0.5, 1.5, n_r) * (r_values[1] - r_values[0])
    L = np.arange(base_lmax + 1, dtype=np.float64)
    C_phi = np.zeros(base_lmax + 1)
    C_phi[1:] = 1e-7 / (L[1:] * (L[1:] + 1.)) ** 2
    C_lens = {k: cl[k].copy() for k in (['TT', 'TE', 'EE', 'BB'] if pol else ['TT'])}
    rr, tt = np.meshgrid(np.linspace(13400., 14200., n_rtau[0]), -np.geomspace(50., 2000., n_rtau[1]),
                         indexing='ij')
    rtau_values = np.stack([rr.ravel(), tt.ravel()], axis=1)
    rtau_w = rng.uniform(0.5, 1.5, len(rtau_values)) * 100.
    return dict(cltot=cltot, cl=cl, beam=beam, mask=mask, k_arr=k_arr,
                Tl_arr=smooth_transfer(2 if pol else 1, k_arr, lmax + 1, seed + 3), r_values=r_values,
                r_weights={t: weights for t in ('gNL-loc', 'gNL-con', 'tauNL-loc')}, rtau_values=rtau_values,
                rtau_weights={t: rtau_w for t in ('gNL-dotdot', 'gNL-dotdel', 'gNL-deldel')}, C_phi=C_phi,
                C_lens_weight=C_lens, lmin=2, lmax=lmax)
