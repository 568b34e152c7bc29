"""The oracle's k-space integral restatement (oracle/shims/k_integrals.py) on the
CPU: j_l' from the recurrence against scipy's derivative, and the (r, tau) and
collider integrals against the golden fixtures made through the reference."""
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_jl_prime_recurrence():
    from scipy.special import spherical_jn
    from oracle.shims import k_integrals as ki
    x = np.linspace(0.5, 80., 41)
    lmin, lmax = 1, 30
    jl = np.stack([spherical_jn(l, x) for l in range(lmin, lmax + 1)])[:, None, :]   # [nl, 1, nx]
    jp = ki.compute_jl_prime(lmin, lmax, 2, 29, jl, 1)
    ref = np.stack([spherical_jn(l, x, derivative=True) for l in range(2, 30)])[:, None, :]
    assert np.abs(jp - ref).max() < 1e-13


@pytest.mark.parametrize("pol", [False, True])
def test_rtau_integrals_match_fixture(pol):
    """The shim's a, b, c and r integrals from the fixture's inputs, on the reference's x grid."""
    from oracle.shims import k_integrals as ki
    d = dict(np.load(os.path.join(GOLD, "tspec_efti_nside16_%s.npz" % ("teb" if pol else "t"))))
    k, T = d["k_arr"], d["Tl_arr"]
    lmin_t, lmax_t = int(d["lmin_t"]), int(d["lmax_t"])
    lmax, lmin = lmax_t + 1, lmin_t - 1
    Pz = 2. * np.pi ** 2. / k ** 3 * 2.1e-9 * (k / 0.05) ** (0.96 - 1)
    npol_out = 3 if pol else 1

    def xgrid(max_kr):
        x = list(np.arange(0, lmax * 2, 0.01)) + list(np.arange(lmax * 2, min(max_kr * 1.01, lmax * 100), 0.1))
        if max_kr > 100 * lmax:
            x += list(np.linspace(lmax * 100, max_kr * 1.01, 1000))
        return np.asarray(x)

    x = xgrid(max(k) * max(d["r_values"]))
    jlx = np.zeros((lmax - lmin + 1, len(x)))
    ki.compute_bessel(x, lmin, lmax, jlx, 1)
    jlkr = ki.interpolate_jlkr(x, k, d["r_values"], jlx, 1)[lmin_t - lmin:lmax_t - lmin + 1]
    out = np.zeros((lmax_t + 1, npol_out, len(d["r_values"])))
    ki.r_integral(k, Pz, T, jlkr, lmin_t, lmax_t, 1, out)
    assert np.abs(out - d["rlXs"]).max() <= 1e-12 * np.abs(d["rlXs"]).max()

    r, tau = d["rtau_values"][:, 0], d["rtau_values"][:, 1]
    x = xgrid(max(k) * (14163.032903769747 + 10000 + 5e6))
    jlx = np.zeros((lmax - lmin + 1, len(x)))
    ki.compute_bessel(x, lmin, lmax, jlx, 1)
    jall = ki.interpolate_jlkr(x, k, r, jlx, 1)
    jprime = ki.compute_jl_prime(lmin, lmax, lmin_t, lmax_t, jall, 1)
    j = jall[lmin_t - lmin:lmax_t - lmin + 1]
    for name, fn, args in (("alXs", ki.a_integral, (k, tau, Pz, T, j)),
                           ("blXs", ki.b_integral, (k, tau, Pz, T, jprime)),
                           ("clXs", ki.c_integral, (k, r, tau, Pz, T, j))):
        out = np.zeros((lmax_t + 1, npol_out, len(r)))
        fn(*args, lmin_t, lmax_t, 1, out)
        assert np.abs(out - d[name]).max() <= 1e-12 * np.abs(d[name]).max(), name


def test_F_integral_hypergeometric_against_mpmath():
    """The oracle's F_L(r, r') (scipy's 2F1) against the same closed form with mpmath's 2F1
    at 40 digits, on the tauNL fixture's radial grid."""
    import mpmath
    from oracle.shims import k_integrals as ki
    d = dict(np.load(os.path.join(GOLD, "tspec_tauloc_nside16_t.npz")))
    r = d["r_values"]
    ns, As, kp = 0.96, 2.1e-9, 0.05
    pref = 2. * np.pi ** 2 * As / kp ** (ns - 1)
    F = np.zeros_like(d["FLLs"])
    ki.compute_F_integral(r, F, 1, F.shape[1] - 1, 0, ns, pref, 1)
    assert np.abs(F - d["FLLs"]).max() <= 1e-14 * np.abs(d["FLLs"]).max()
    mpmath.mp.dps = 40
    for L in (1, 2, 7, 20, 47):
        for i, j in ((0, 0), (0, 1), (2, 5), (4, 3)):
            ri, rj = (r[i], r[j]) if r[i] <= r[j] else (r[j], r[i])
            i1, i2, i3 = L + (ns - 1.) / 2., (ns - 2.) / 2., L + 1.5
            pf = 2. ** (ns - 3) * pref * mpmath.exp(mpmath.loggamma(i1) - mpmath.loggamma(1 - i2) - mpmath.loggamma(i3))
            exact = float(pf * mpmath.hyp2f1(i1, i2, i3, (mpmath.mpf(ri) / rj) ** 2) * (mpmath.mpf(ri) / rj) ** L
                          * mpmath.mpf(rj) ** (1 - ns))
            assert abs(F[0, L, i, j] - exact) <= 1e-11 * abs(exact), (L, i, j)


def test_F_integral_shifted_against_mpmath():
    """The oracle's F_{L,L+n}(r, r') for n = -2..2 (nmax_F = 2, the direction-dependent tauNL
    fixture's radial grid and L range) against its closed form with mpmath's 2F1 at 40 digits,
    for r <= r' (argument r^2/r'^2, power L) and r > r' (argument r'^2/r^2, power L + n)."""
    import mpmath
    from oracle.shims import k_integrals as ki
    d = dict(np.load(os.path.join(GOLD, "tspec_direc_nside16_t.npz")))
    r = d["r_values"]
    ns, As, kp = 0.96, 2.1e-9, 0.05
    pref = 2. * np.pi ** 2 * As / kp ** (ns - 1)
    F = np.zeros_like(d["FLLs"])
    ki.compute_F_integral(r, F, 2, 40, 2, ns, pref, 1)
    assert np.abs(F - d["FLLs"]).max() <= 1e-14 * np.abs(d["FLLs"]).max()
    mpmath.mp.dps = 40
    for n in (-2, -1, 1, 2):
        for L in (3, 9, 33):  # the reference leaves F = 0 where L + n < 1
            for i, j in ((0, 0), (0, 3), (4, 1)):
                ri, rj = mpmath.mpf(r[i]), mpmath.mpf(r[j])
                i1 = L + (n - 1. + ns) / 2.
                if ri <= rj:
                    i2, i3, x, pw, big = (ns - 2 - n) / 2., L + 1.5, (ri / rj) ** 2, (ri / rj) ** L, rj
                else:
                    i2, i3, x, pw, big = (ns - 2 + n) / 2., L + n + 1.5, (rj / ri) ** 2, (rj / ri) ** (L + n), ri
                pf = 2. ** (ns - 3) * pref * mpmath.exp(mpmath.loggamma(i1) - mpmath.loggamma(1 - i2)
                                                        - mpmath.loggamma(i3))
                exact = float(pf * mpmath.hyp2f1(i1, i2, i3, x) * pw * big ** (1 - ns))
                assert abs(F[2 + n, L, i, j] - exact) <= 1e-11 * abs(exact), (n, L, i, j)


def test_collider_integrals_match_fixture():
    """The shim's collider p^beta and F^beta integrals (collider_p_integral, compute_collider_F_integral) from the
    collider fixture's inputs, on the reference's grids (polyspec/tspec_template.py:536-703), T only: beta =
    nu_s - 3/2 for the light particles and -3/2 - i mu_s for the heavy ones (Im beta > 0 is not stored)."""
    from oracle.shims import k_integrals as ki
    d = dict(np.load(os.path.join(GOLD, "tspec_collider_nside16_t.npz")))
    k, T, r = d["k_arr"], d["Tl_arr"], d["r_values"]
    lmin_t, lmax_t, Lmin, Lmax, K_coll = 2, 30, 2, 40, 0.01
    Pzeta = lambda kk: 2. * np.pi ** 2. / kk ** 3 * 2.1e-9 * (kk / 0.05) ** (0.96 - 1)
    params = {-0.8: [[0, 0]], -1.2: [[1, 0], [1, 2]], -1.5: [[1, 0], [1, 2]], -1.5 - 0.5j: [[0, 0]],
              -1.5 - 0.8j: [[1, 0], [1, 2]]}
    nmax_coll, nmax_coll_F = 1, 2
    lmax = max(lmax_t + 1, lmax_t + nmax_coll)
    lmin = max(min(lmin_t - 1, lmin_t - nmax_coll), 0)
    max_kr = max(k) * max(r)
    x = np.asarray(list(np.arange(0, lmax * 2, 0.01)) + list(np.arange(lmax * 2, min(max_kr * 1.01, lmax * 100), 0.1)))
    jlx = np.zeros((lmax - lmin + 1, len(x)))
    ki.compute_bessel(x, lmin, lmax, jlx, 1)
    jall = ki.interpolate_jlkr(x, k, r, jlx, 1)
    for beta, pr in params.items():
        nm = max(p[0] for p in pr)
        out = np.zeros((2 * nm + 1, lmax + 1, 1, len(r)), dtype=np.complex128)
        ki.collider_p_integral(k, Pzeta(k), T, jall, beta, K_coll, lmin_t, lmax_t, lmin, lmax, nm, 1, out)
        ref = d["coll_plLXs_%.8f,%.8f" % (np.real(beta), np.imag(beta))]
        assert np.abs(out - ref).max() <= 1e-12 * np.abs(ref).max(), beta
    K = np.geomspace(0.1 / (14163.032903769747 + 5000), K_coll * 1.01, 5000)
    Lt_max, Lt_min = Lmax + nmax_coll_F, max(Lmin - nmax_coll_F, 0)
    y = np.asarray(list(np.arange(0, Lt_max * 2, 0.01)) + list(np.arange(Lt_max * 2, K_coll * max(r) * 1.01, 0.01)))
    jly = np.zeros((Lt_max - Lt_min + 1, len(y)))
    ki.compute_bessel(y, Lt_min, Lt_max, jly, 1)
    jlK = ki.interpolate_jlkr(y, K, r, jly, 1)
    for beta, pr in params.items():
        nF = max(p[1] for p in pr)
        out = np.zeros((2 * nF + 1, 48, len(r), len(r)), dtype=np.complex128)
        ki.compute_collider_F_integral(K, Pzeta(K), jlK, -2. * beta, K_coll, Lmin, Lmax, nF, nmax_coll_F, 1, out)
        ref = d["coll_FLLs_%.8f,%.8f" % (np.real(beta), np.imag(beta))]
        assert np.abs(out - ref).max() <= 1e-12 * np.abs(ref).max(), beta
