"""ORACLE shim: numpy restatement of the reference's k-space integrals
(polyspec/cython/k_integrals.pyx), standing in for the compiled module, which
links GSL (absent here).  Test infrastructure only.

Restated (same grids, branches and trapezium rule, vectorised):
  * compute_bessel        k_integrals.pyx:28-71   j_l(x) table; GSL's Steed
                          recurrence (gsl_sf_bessel_jl_steed_array, GSL version
                          unpinned by the reference) is replaced by scipy's
                          spherical_jn, with the reference's branches kept: x = 0,
                          the large-x limit for x > 18000 + lmax, and zeros where
                          the small-x limit falls below 1e-150;
  * interpolate_jlkr      :84-110  linear interpolation of the table to k r;
  * q_integral            :312-353 q_l^X(r) = (-1)^l Sum_k dk (f_k + f_k+1),
                          f = (2/pi) k^2 / 2 T_l^X(k) j_l(kr);
  * p_integral            :262-310 the same with P_zeta(k) in f and j_{l+n};
  * r_integral            :355-396 f = (2/pi) k^2 / 2 P_zeta(k)^(3/4) T_l^X(k) j_l(kr);
  * compute_jl_prime      :112-124 j_l' = (l j_{l-1} - (l+1) j_{l+1}) / (2l+1);
  * a_integral            :127-170 f = (2/pi) k^(13/4) P_zeta^(3/4) / 2 e^(k tau) T j_l(kr);
  * b_integral            :172-215 f = (2/pi) k^(9/4) P_zeta^(3/4) / 2 (1 - k tau) e^(k tau) T j_l'(kr);
  * c_integral            :217-260 f = (2/pi) k^(5/4) P_zeta^(3/4) / 2 (1 - k tau) e^(k tau) / r
                          T j_l(kr), the sum weighted by sqrt(l (l+1)).
  * compute_F_integral    :453-494 F_{L,L+n}(r, r') in closed form; GSL's lngamma and
                          hyperg_2F1 (GSL version unpinned by the reference) are
                          replaced by scipy's gammaln and hyp2f1.
  * collider_p_integral   :399-451 p_integral's sum with kprod = (2/pi) k^(2+beta) P_zeta / 2
                          (complex) for k >= k_coll;
  * compute_collider_F_integral :496-545 F^{betaF}_{L,L+n}(r, r') by the trapezium rule
                          over K <= K_coll, kprod = (2/pi) K^(2+betaF) P_zeta / 2.
"""
import numpy as np
from scipy.special import gammaln, hyp2f1, spherical_jn


def _smallx(l, x):
    """x << l limit of j_l(x) (k_integrals.pyx:73-75)."""
    return (np.e * x / (2. * l + 1.)) ** (l + 0.5) / np.sqrt(4 * x * (l + 0.5))


def compute_bessel(x_arr, lmin, lmax, jlx_arr, nthreads):
    x_arr = np.asarray(x_arr, dtype=np.float64)
    nx = len(x_arr)
    tmp = np.zeros((nx, lmax + 1))
    ls = np.arange(lmax + 1)
    small = 1e-150
    with np.errstate(over='ignore', under='ignore', divide='ignore', invalid='ignore'):
        for ix in range(nx):
            x = x_arr[ix]
            if x == 0.:
                tmp[ix, 0] = 1.
            elif x > 18000 + lmax:
                tmp[ix] = np.sin(x - ls * np.pi / 2.) / x
            else:
                if abs(_smallx(lmax, x)) > small:
                    lt = lmax
                else:
                    lt = lmax
                    for l in range(lmax, 0, -1):
                        lt = l
                        if abs(_smallx(l, x)) > small:
                            break
                    else:
                        lt = 1  # the reference's loop variable ends at 1 when nothing breaks
                tmp[ix, :lt + 1] = spherical_jn(np.arange(lt + 1), x)
    jlx_arr[:, :] = tmp[:, lmin:lmax + 1].T


def interpolate_jlkr(x_arr, k_arr, r_arr, jlx_arr, nthreads):
    x_arr = np.asarray(x_arr)
    kr = np.asarray(k_arr)[None, :] * np.asarray(r_arr)[:, None]          # [nr, nk]
    # k r beyond the last grid point (the collider F set-up's K grid ends at 1.01 K_coll, past its y
    # grid) reads past the reference's table; its integrand prefactor is zero there, so the clamped
    # extrapolation stands in for it
    ix = np.minimum(np.searchsorted(x_arr, kr) - 1, len(x_arr) - 2)
    dx = x_arr[ix + 1] - x_arr[ix]
    xp = (x_arr[ix + 1] - kr) / dx
    xm = (kr - x_arr[ix]) / dx
    jl = np.asarray(jlx_arr)
    return jl[:, ix] * xp[None] + jl[:, ix + 1] * xm[None]               # [nl, nr, nk]


def _trapz(kprod, T, jl, k_arr):
    """Sum_k (k_{i} - k_{i-1}) (f_{i-1} + f_i), f = kprod T jl, over the last axis."""
    f = kprod * T * jl
    dk = np.diff(k_arr)
    return np.sum(dk * (f[..., :-1] + f[..., 1:]), axis=-1)


def q_integral(k_arr, Tl_arr, jlkr, lmin, lmax, nthreads, integs):
    k_arr = np.asarray(k_arr)
    kprod = 2. / np.pi * k_arr * k_arr / 2.
    for il in range(lmax + 1 - lmin):
        l = lmin + il
        for X in range(len(Tl_arr)):
            integs[l, X, :] += (-1.) ** l * _trapz(kprod, np.asarray(Tl_arr)[X, l][None], jlkr[il], k_arr)


def p_integral(k_arr, Pzeta_arr, Tl_arr, jlkr_all, lmin, lmax, arr_lmin, arr_lmax, this_nmax, nthreads, integs):
    k_arr = np.asarray(k_arr)
    kprod = 2. / np.pi * k_arr * k_arr * np.asarray(Pzeta_arr) / 2.
    nmax = len(integs) // 2
    for n in range(-this_nmax, this_nmax + 1):
        lshift1 = min(0, lmin - arr_lmin + n)
        lshift2 = max(0, lmin - arr_lmin + n)
        for il in range(lmax - lmin + lshift1 + 1):
            l = lmin - lshift1 + il
            for X in range(len(Tl_arr)):
                integs[nmax + n, l, X, :] += (-1.) ** l * _trapz(kprod, np.asarray(Tl_arr)[X, l][None],
                                                                 jlkr_all[lshift2 + il], k_arr)


def r_integral(k_arr, Pzeta_arr, Tl_arr, jlkr, lmin, lmax, nthreads, integs):
    k_arr = np.asarray(k_arr)
    kprod = 2. / np.pi * k_arr * k_arr / 2. * np.asarray(Pzeta_arr) ** (3. / 4.)
    for il in range(lmax + 1 - lmin):
        l = lmin + il
        for X in range(len(Tl_arr)):
            integs[l, X, :] += (-1.) ** l * _trapz(kprod, np.asarray(Tl_arr)[X, l][None], jlkr[il], k_arr)


def compute_jl_prime(lmin, lmax, lmin_base, lmax_base, jls, nthreads):
    jls = np.asarray(jls)
    out = np.zeros((lmax_base - lmin_base + 1,) + jls.shape[1:])
    for l in range(lmin_base, lmax_base + 1):
        out[l - lmin_base] = (l * jls[l - lmin - 1] - (l + 1.) * jls[l - lmin + 1]) / (2. * l + 1.)
    return out


def _ktau(k_arr, tau_arr, Pzeta_arr, kpow, damped, r_arr=None):
    """[ntau, nk] k- and tau-dependent factor of the a, b, c integrands."""
    k_arr, tau = np.asarray(k_arr), np.asarray(tau_arr)
    kpref = 2. / np.pi * k_arr ** kpow * np.asarray(Pzeta_arr) ** (3. / 4.) / 2.
    kt = k_arr[None, :] * tau[:, None]
    out = kpref[None, :] * (1. - kt) * np.exp(kt) if damped else kpref[None, :] * np.exp(kt)
    if r_arr is not None:
        out = out / np.asarray(r_arr)[:, None]
    return out


def _rtau_integral(k_arr, ktauprod, Tl_arr, jl, lmin, lmax, integs, lweight):
    for il in range(lmax + 1 - lmin):
        l = lmin + il
        pref = (-1.) ** l * (np.sqrt(l * (l + 1.)) if lweight else 1.)
        for X in range(len(Tl_arr)):
            integs[l, X, :] += pref * _trapz(ktauprod, np.asarray(Tl_arr)[X, l][None], jl[il], np.asarray(k_arr))


def a_integral(k_arr, tau_arr, Pzeta_arr, Tl_arr, jlkrtau, lmin, lmax, nthreads, integs):
    _rtau_integral(k_arr, _ktau(k_arr, tau_arr, Pzeta_arr, 13. / 4., False), Tl_arr, jlkrtau, lmin, lmax, integs,
                   False)


def b_integral(k_arr, tau_arr, Pzeta_arr, Tl_arr, jlkrtau_prime, lmin, lmax, nthreads, integs):
    _rtau_integral(k_arr, _ktau(k_arr, tau_arr, Pzeta_arr, 9. / 4., True), Tl_arr, jlkrtau_prime, lmin, lmax,
                   integs, False)


def c_integral(k_arr, r_arr, tau_arr, Pzeta_arr, Tl_arr, jlkrtau, lmin, lmax, nthreads, integs):
    _rtau_integral(k_arr, _ktau(k_arr, tau_arr, Pzeta_arr, 5. / 4., True, r_arr), Tl_arr, jlkrtau, lmin, lmax,
                   integs, True)


def compute_F_integral(r_arr, FLLs, Lmin, Lmax, nmax_F, ns, _pref, nthreads):
    r_arr = np.asarray(r_arr, dtype=np.float64)
    pref = 2. ** (ns - 3) * _pref
    for n in range(-nmax_F, nmax_F + 1):
        i2a, i2b = (ns - 2 - n) / 2., (ns - 2 + n) / 2.
        lgam2a, lgam2b = gammaln(1. - i2a), gammaln(1. - i2b)
        for L in range(max(Lmin - nmax_F, 0), Lmax + nmax_F + 1):
            if L + n < 1 or L < 1 or L + n > Lmax + nmax_F:
                continue
            i1, i3a, i3b = L + (n - 1. + ns) / 2., L + 1.5, L + n + 1.5
            lgam1 = gammaln(i1)
            prefa = pref * np.exp(lgam1 - lgam2a - gammaln(i3a))
            prefb = pref * np.exp(lgam1 - lgam2b - gammaln(i3b))
            for ir, ri in enumerate(r_arr):
                for jr, rj in enumerate(r_arr):
                    if ri <= rj:
                        FLLs[nmax_F + n, L, ir, jr] = prefa * hyp2f1(i1, i2a, i3a, ri * ri / (rj * rj)) \
                            * (ri / rj) ** L * rj ** (1. - ns)
                    else:
                        FLLs[nmax_F + n, L, ir, jr] = prefb * hyp2f1(i1, i2b, i3b, rj * rj / (ri * ri)) \
                            * (rj / ri) ** (L + n) * ri ** (1. - ns)


def collider_p_integral(k_arr, Pzeta_arr, Tl_arr, jlkr_all, beta, k_coll, lmin, lmax, arr_lmin, arr_lmax,
                        this_nmax, nthreads, integs):
    """p_lL^{beta,X}(r) (k_integrals.pyx:399-451): p_integral's sum with the complex
    kprod = (2/pi) k^(2 + beta) P_zeta(k) / 2 for k >= k_coll, zero below."""
    k_arr = np.asarray(k_arr)
    kprod = np.where(k_arr >= k_coll, 2. / np.pi * k_arr.astype(np.complex128) ** (2. + beta)
                     * np.asarray(Pzeta_arr) / 2., 0.)
    for n in range(-this_nmax, this_nmax + 1):
        lshift1 = min(0, lmin - arr_lmin + n)
        lshift2 = max(0, lmin - arr_lmin + n)
        for il in range(lmax - lmin + lshift1 + 1):
            l = lmin - lshift1 + il
            for X in range(len(Tl_arr)):
                integs[this_nmax + n, l, X, :] += (-1.) ** l * _trapz(kprod, np.asarray(Tl_arr)[X, l][None],
                                                                      jlkr_all[lshift2 + il], k_arr)


def compute_collider_F_integral(K_arr, Pzeta_arr, jlK, betaF, K_coll, Lmin, Lmax, this_nmax_F, coll_nmax_F,
                                nthreads, integs):
    """F^{-2 beta}_{L,L+n}(r, r') (k_integrals.pyx:496-545): Sum_K dK (f_{K-1} + f_K),
    f = (2/pi) K^(2 + betaF) P_zeta(K) / 2 j_L(K r) j_{L+n}(K r') for K <= K_coll (zero above),
    with j from the interpolated [L - max(Lmin - coll_nmax_F, 0), r, K] table; n = 0 is
    filled symmetrically from r' <= r."""
    K_arr = np.asarray(K_arr)
    Kprod = np.where(K_arr <= K_coll, 2. / np.pi * K_arr.astype(np.complex128) ** (2. + betaF)
                     * np.asarray(Pzeta_arr) / 2., 0.)
    jlK = np.asarray(jlK)
    global_Lmin = max(Lmin - coll_nmax_F, 0)
    dK = np.diff(K_arr)
    for n in range(-this_nmax_F, this_nmax_F + 1):
        for L in range(max(Lmin - this_nmax_F, 0), Lmax + this_nmax_F + 1):
            if L + n < 1 or L < 1 or L + n > Lmax + this_nmax_F:
                continue
            ind1, ind2 = L - global_Lmin, L - global_Lmin + n
            f = Kprod[None, None, :] * jlK[ind1][:, None, :] * jlK[ind2][None, :, :]
            tmp = np.sum(dK * (f[..., :-1] + f[..., 1:]), axis=-1)
            if n == 0:
                tmp = np.tril(tmp) + np.tril(tmp, -1).T
            integs[this_nmax_F + n, L] = tmp
