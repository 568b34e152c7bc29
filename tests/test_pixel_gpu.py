"""libpscuda pixel products, radial sums, harmonic weightings and the Fisher
outer product against the CPU oracle (numpy restatement of the reference's
Cython kernels) and, where oracle/_ref is built, the compiled reference itself.

Tolerances (FP64 throughout): 1e-14 of the largest magnitude for elementwise
products (one or two roundings, FMA contraction may differ), 1e-12 relative for
the radial pixel sums and the outer product (different summation order)."""
import os
import sys

import numpy as np
import pytest

import pixel_cases as C

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
from oracle import pixel as O  # noqa: E402


def close(a, b, tol):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape, (a.shape, b.shape)
    if a.size == 0:
        return True
    return np.max(np.abs(a - b)) <= tol * max(np.max(np.abs(b)), 1e-300)


def _ref():
    d = os.path.join(ROOT, "oracle", "_ref")
    if d not in sys.path:
        sys.path.insert(0, d)
    try:
        import tauNL_utils as T
        import ideal_fisher as F
        return T, F
    except ImportError:
        return None, None


@pytest.mark.gpu
@pytest.mark.parametrize("op", sorted(C.PRODUCTS))
@pytest.mark.parametrize("shape", [(3, 1001), (1, 5), (24, 12 * 32 ** 2), (2, 0)])
def test_products(op, shape):
    from polyspec_b200 import pixel as P
    kinds, fac = C.PRODUCTS[op]
    xs = C.maps(kinds, shape, seed=sum(map(ord, op)) + shape[1])
    extra = () if fac is None else (fac,)
    if op in C.TAUNL_PRODUCTS:
        out = getattr(P.tauNL_utils(*C.taunl_args(shape[0], 8)), op)(*xs)
    else:
        out = getattr(P, op)(*xs, *extra)
    assert close(out, getattr(O, op)(*xs, *extra), 1e-14)
    T, F = _ref()
    if T is not None and shape[1] > 0:
        ref = (getattr(T.tauNL_utils(*C.taunl_args(shape[0], 8)), op)(*xs) if op in C.TAUNL_PRODUCTS
               else getattr(F, op)(*xs, *extra, 2))
        assert close(out, ref, 1e-14)


@pytest.mark.gpu
def test_products_stay_on_device():
    import torch
    from polyspec_b200 import pixel as P
    a, b = (torch.randn(4, 999, dtype=torch.float64, device="cuda") for _ in range(2))
    c = torch.randn(4, 999, dtype=torch.complex128, device="cuda")
    out = P.multiplyRC(a, c)
    assert isinstance(out, torch.Tensor) and out.is_cuda
    assert torch.allclose(out, a * c, rtol=0, atol=1e-14 * float(out.abs().max()))
    t = P.tauNL_utils(*C.taunl_args(4, 8))
    assert torch.allclose(t.multiply2R(a, b), a * b, rtol=0, atol=1e-14 * float((a * b).abs().max()))


@pytest.mark.gpu
@pytest.mark.parametrize("kind", sorted(C.SUMS))
@pytest.mark.parametrize("nr,npix", [(5, 3001), (1, 7), (24, 12 * 64 ** 2)])
def test_radial_sums(kind, nr, npix):
    from polyspec_b200 import pixel as P
    kinds, has_tau = C.SUMS[kind]
    xs = C.maps(kinds, (nr, npix), seed=nr * 7 + npix)
    rng = np.random.default_rng(nr)
    w, tau = rng.normal(size=nr), rng.uniform(0.5, 2.0, size=nr)
    args = (w, tau) if has_tau else (w,)
    t = P.tauNL_utils(*C.taunl_args(nr, 8))
    got = getattr(t, kind)(*args, *xs)
    want = getattr(O, kind)(*args, *xs)
    scale = getattr(O, kind)(*[np.abs(a) for a in args], *[np.abs(x) for x in xs])
    assert abs(got - want) <= 1e-12 * scale
    # fixed-order reduction: repeated calls agree bit for bit
    assert getattr(t, kind)(*args, *xs) == got
    T, _ = _ref()
    if T is not None:
        ref = getattr(T.tauNL_utils(*C.taunl_args(nr, 8)), kind)(*args, *xs)
        assert abs(got - ref) <= 1e-12 * scale


@pytest.mark.gpu
@pytest.mark.parametrize("npol,npix", [(1, 777), (3, 777), (3, 12 * 64 ** 2)])
def test_lens_phi(npol, npix):
    from polyspec_b200 import pixel as P
    U, V, U2, V2 = C.maps("cccc", (npol, npix), seed=npol + npix)
    assert close(P.lens_phi_sum(U, V), O.lens_phi_sum(U, V), 1e-14)
    assert close(P.lens_phi_sum_sym(U, U2, V, V2), O.lens_phi_sum_sym(U, U2, V, V2), 1e-14)
    _, F = _ref()
    if F is not None:
        assert close(P.lens_phi_sum(U, V), F.lens_phi_sum(U, V, 2), 1e-14)
        assert close(P.lens_phi_sum_sym(U, U2, V, V2), F.lens_phi_sum_sym(U, U2, V, V2, 2), 1e-14)


@pytest.mark.gpu
@pytest.mark.parametrize("npol", [1, 2, 3])
@pytest.mark.parametrize("lmax,nr", [(12, 7), (100, 24)])
def test_harmonic_weightings(npol, lmax, nr):
    from polyspec_b200 import pixel as P
    l, m = C.lm_setup(lmax)
    rng = np.random.default_rng(npol * 100 + lmax)
    flX = rng.normal(size=(lmax + 1, npol, nr))
    h = rng.normal(size=(npol, len(l))) + 1j * rng.normal(size=(npol, len(l)))
    t = P.tauNL_utils(*C.taunl_args(nr, lmax))
    assert close(t.apply_fl_weights(flX, h, 0.3), O.apply_fl_weights(l, flX, h, 0.3), 1e-14)
    lm_map = rng.normal(size=(nr, len(l))) + 1j * rng.normal(size=(nr, len(l)))
    w = rng.normal(size=nr)
    assert close(t.radial_sum(lm_map, w, flX), O.radial_sum(l, lm_map, w, flX), 1e-12)
    lm2 = rng.normal(size=(2, nr, len(l))) + 1j * rng.normal(size=(2, nr, len(l)))
    assert close(t.radial_sum_spin1(lm2, w, flX), O.radial_sum_spin1(l, lm2, w, flX), 1e-12)
    T, _ = _ref()
    if T is not None:
        r = T.tauNL_utils(*C.taunl_args(nr, lmax))
        assert close(t.apply_fl_weights(flX, h, 0.3), r.apply_fl_weights(flX, h, 0.3), 1e-14)
        assert close(t.radial_sum(lm_map, w, flX), r.radial_sum(lm_map, w, flX), 1e-12)
        assert close(t.radial_sum_spin1(lm2, w, flX), r.radial_sum_spin1(lm2, w, flX), 1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("sym", [False, True])
@pytest.mark.parametrize("na,nb,nin", [(6, 9, 500), (1, 1, 3), (37, 37, 20011), (16, 17, 4096)])
def test_outer_product(sym, na, nb, nin):
    from polyspec_b200 import pixel as P
    if sym:
        nb = na
    rng = np.random.default_rng(na * nb + nin)
    Qa = rng.normal(size=(4, na, nin)) + 1j * rng.normal(size=(4, na, nin))
    Qb = Qa if sym else rng.normal(size=(4, nb, nin)) + 1j * rng.normal(size=(4, nb, nin))
    got = P.outer_product(Qa, Qb, 0, sym)
    assert close(got, O.outer_product(Qa, Qb, sym), 1e-12)
    if sym:
        assert np.array_equal(got, got.T)
    _, F = _ref()
    if F is not None:
        assert close(got, F.outer_product(Qa, Qb, 2, sym), 1e-12)


def _tau_case(nr, seed, zero_w=True):
    """Random (L, M) maps, F_L(r, r') and radial weights (some zero) for the local-tauNL kernels."""
    from pixel_cases import lm_setup
    rng = np.random.default_rng(seed)
    base_lmax, Lmin, Lmax = 20, 2, 12
    l, m = lm_setup(base_lmax)
    sel = l <= Lmax
    Lfull, Mfull = l[sel], m[sel]
    filt = Lfull >= Lmin
    X = rng.normal(size=(nr, sel.sum())) + 1j * rng.normal(size=(nr, sel.sum()))
    A = rng.normal(size=(nr, sel.sum())) + 1j * rng.normal(size=(nr, sel.sum()))
    F = rng.normal(size=(1, Lmax + 1, nr, nr))
    F = F + np.swapaxes(F, 2, 3)   # F_L(r, r') is symmetric for n = 0
    w = rng.uniform(0.5, 2.0, nr)
    if zero_w and nr > 2:
        w[1] = 0.
    lm_L = np.where(filt, Lfull, -1).astype(np.int32)
    lm_w = np.where(Mfull == 0, 1., 2.)
    args = (1, nr, l.astype(np.int32), m.astype(np.int32), Lmin, Lmax, l.astype(np.int32), m.astype(np.int32),
            Lfull[filt].astype(np.int32), Mfull[filt].astype(np.int32), 0)
    return X, A, F, w, lm_L, lm_w, filt, args


@pytest.mark.gpu
@pytest.mark.parametrize("nr,seed", [(1, 1), (6, 2), (24, 3), (97, 4)])
def test_tau_convolve_and_sum(nr, seed):
    """ps_tau_convolve_F against the compiled reference's convolve_F_n000 and tau_sum_n0
    (zero radial weights included): 1e-13 of the largest magnitude."""
    import torch
    from polyspec_b200 import pixel as P
    T, _ = _ref()
    if T is None:
        pytest.skip("oracle/_ref is not built")
    X, A, F, w, lm_L, lm_w, filt, args = _tau_case(nr, seed)
    dev = torch.device("cuda")
    tX, tA, tF = (torch.as_tensor(v, device=dev) for v in (X, A, F[0]))
    out = P.tau_convolve_F(tX, torch.as_tensor(lm_L, device=dev), tF, w).cpu().numpy()
    ut = T.tauNL_utils(*args)
    ref = np.zeros((len(filt), nr), dtype=np.complex128)
    ut.convolve_F_n000(np.ascontiguousarray(X[:, filt].T), F, w, ref, 0, np.arange(nr, dtype=np.int32))
    assert close(out.T, ref, 1e-13)
    tau = P.tau_convolve_F(tX, torch.as_tensor(lm_L, device=dev), tF, w, A=tA,
                           lm_w=torch.as_tensor(lm_w, device=dev))
    tau_ref = ut.tau_sum_n0(np.ascontiguousarray(A[:, filt].T)[None], np.ascontiguousarray(X[:, filt].T)[None],
                            F[0], w, 0)
    assert abs(tau - tau_ref) <= 1e-12 * abs(tau_ref)


@pytest.mark.gpu
@pytest.mark.parametrize("nr,seed", [(6, 5), (24, 6)])
def test_tau_reference_signatures(nr, seed):
    """The reference-signature tauNL_utils.tau_sum_n0 / convolve_F_n000 (with a subset of radial
    indices) and the module functions compute_productP_real_all, compute_productQ_real_all and
    integrate_pq against the compiled reference: 1e-13 of the largest magnitude."""
    from polyspec_b200 import pixel as P
    T, Fm = _ref()
    if T is None:
        pytest.skip("oracle/_ref is not built")
    X, A, F, w, lm_L, lm_w, filt, args = _tau_case(nr, seed)
    ut, mine = T.tauNL_utils(*args), P.tauNL_utils(*args)
    a1 = np.ascontiguousarray(A[:, filt].T)[None]
    a2 = np.ascontiguousarray(X[:, filt].T)[None]
    t_ref, t = ut.tau_sum_n0(a1, a2, F[0], w, 0), mine.tau_sum_n0(a1, a2, F[0], w, 0)
    assert abs(t - t_ref) <= 1e-12 * abs(t_ref)
    inds = np.arange(nr, dtype=np.int32)[::2].copy()
    PQ = np.ascontiguousarray(a2[0][:, inds])
    out_ref = np.zeros((len(filt), len(inds)), dtype=np.complex128)
    out = np.zeros_like(out_ref)
    ut.convolve_F_n000(PQ, F, w[:len(inds)].copy(), out_ref, 0, inds)
    mine.convolve_F_n000(PQ, F, w[:len(inds)].copy(), out, 0, inds)
    assert close(out, out_ref, 1e-13)
    rng = np.random.default_rng(seed)
    npix = 768
    Pm = rng.normal(size=(2, nr, npix))
    Fq = rng.normal(size=(3, nr, npix)) + 1j * rng.normal(size=(3, nr, npix))
    for wts, pq, fi in (([12.], [0], [0]), ([4., 4.], [1, 0], [0, 2])):
        wts, pq, fi = np.asarray(wts), np.asarray(pq, dtype=np.int32), np.asarray(fi, dtype=np.int32)
        assert close(P.compute_productP_real_all(Pm, Fq, wts, pq, fi, 1),
                     Fm.compute_productP_real_all(Pm, Fq, wts, pq, fi, 1), 1e-14)
        assert close(P.compute_productQ_real_all(Pm, Fq[:, None], wts, pq, fi, 0, 1),
                     Fm.compute_productQ_real_all(Pm, np.ascontiguousarray(Fq[:, None]), wts, pq, fi, 0, 1), 1e-14)
    lmax = 15
    from pixel_cases import lm_setup
    ls = lm_setup(lmax)[0].astype(np.int64)
    flX = rng.normal(size=(lmax + 1, 2, nr))
    Pf = rng.normal(size=(len(ls), len(inds))) + 1j * rng.normal(size=(len(ls), len(inds)))
    o_ref = np.zeros((2, len(ls)), dtype=np.complex128)
    o = np.zeros_like(o_ref)
    Fm.integrate_pq(flX, Pf, ls, w[:len(inds)].copy(), o_ref, inds, 1)
    P.integrate_pq(flX, Pf, ls, w[:len(inds)].copy(), o, inds, 1)
    assert close(o, o_ref, 1e-13)


@pytest.mark.gpu
@pytest.mark.parametrize("n,mu,npol,lmax", [(1, 0, 1, 12), (1, 1, 2, 12), (2, 0, 2, 12), (3, 2, 2, 12), (3, 3, 1, 12),
                                             (2, 1, 2, 60), (5, 4, 2, 40)])
def test_shift_and_weight_map_all(n, mu, npol, lmax):
    """Gaunt-weighted l-shifts (ps_shift_weight_map_all) against the compiled reference's
    shift_and_weight_map_all, accumulated into non-zero arrays: 1e-13 of the largest magnitude."""
    from polyspec_b200 import pixel as P
    from pixel_cases import lm_setup
    T, _ = _ref()
    if T is None:
        pytest.skip("oracle/_ref is not built")
    rng = np.random.default_rng(n * 100 + mu * 10 + npol + lmax)
    base_lmax, lmin, nmax, nr = lmax + 6, 2, max(n, 3) + 1, 3
    l, m = lm_setup(base_lmax)
    sel = (l >= lmin) & (l <= lmax)
    ls, ms = l[sel].astype(np.int32), m[sel].astype(np.int32)
    flX = rng.normal(size=(2 * nmax + 1, base_lmax + 1, npol, nr))
    h = rng.normal(size=(npol, len(ls))) + 1j * rng.normal(size=(npol, len(ls)))
    weight = 0.7 - 0.3j
    nt = (lmax + n + 1) * (lmax + n + 2) // 2
    L0 = rng.normal(size=(nr, nt)) + 1j * rng.normal(size=(nr, nt))
    Lr, Li = L0.copy(), 2. * L0
    args = (1, nr, l.astype(np.int32), m.astype(np.int32), 1, 2 * lmax, ls, ms, ls, ms, nmax)
    T.tauNL_utils(*args).shift_and_weight_map_all(flX, h, n, mu, weight, Lr, Li, nmax)
    Gr, Gi = L0.copy(), 2. * L0
    P.tauNL_utils(*args).shift_and_weight_map_all(flX, h, n, mu, weight, Gr, Gi, nmax)
    assert close(Gr, Lr, 1e-13) and close(Gi, Li, 1e-13)


def _general_case(nr, nmax_F, seed, lmax_L=11, Lmin=2, Lmax=9):
    from pixel_cases import lm_setup
    rng = np.random.default_rng(seed)
    l, m = lm_setup(lmax_L + 4)
    sel = (l >= 1) & (l <= lmax_L)
    Ls, Ms = l[sel].astype(np.int32), m[sel].astype(np.int32)
    F = rng.normal(size=(2 * nmax_F + 1, Lmax + 3, nr, nr))
    w = rng.uniform(0.5, 1.5, size=nr)
    w[nr // 2] = 0.
    args = (1, nr, l.astype(np.int32), m.astype(np.int32), Lmin, Lmax, Ls, Ms, Ls, Ms, nmax_F)
    return rng, Ls, F, w, args, int(np.sum(l <= lmax_L))


@pytest.mark.gpu
@pytest.mark.parametrize("n1,n3,n", [(1, 1, 0), (1, 1, 2), (1, 2, 1), (2, 1, 3), (2, 2, 2), (3, 2, 1)])
def test_tau_general(n1, n3, n):
    """tauNL_utils.tau_sum_general and convolve_F_general (every mu1, a subset of radial indices,
    accumulated into non-zero outputs) against the compiled reference: 1e-12 relative for the sum,
    1e-13 of the largest magnitude for the convolutions."""
    from polyspec_b200 import pixel as P
    T, _ = _ref()
    if T is None:
        pytest.skip("oracle/_ref is not built")
    nr = 5
    rng, Ls, F, w, args, nfull = _general_case(nr, max(n, 3), 100 * n1 + 10 * n3 + n)
    ut, mine = T.tauNL_utils(*args), P.tauNL_utils(*args)

    def cplx(*shape):
        return rng.normal(size=shape) + 1j * rng.normal(size=shape)

    a1, a2 = cplx(2 * n1 + 1, len(Ls), nr), cplx(2 * n3 + 1, len(Ls), nr)
    t_ref, t = ut.tau_sum_general(a1, a2, F, w, n1, n3, n), mine.tau_sum_general(a1, a2, F, w, n1, n3, n)
    assert abs(t - t_ref) <= 1e-12 * max(abs(t_ref), 1e-300), (t, t_ref)
    inds = np.array([0, 2, 3, 4], dtype=np.int32)
    PQ = cplx(2 * n3 + 1, len(Ls), len(inds))
    for mu1 in range(-n1, n1 + 1):
        o0r, o0i = cplx(nfull, len(inds)), cplx(nfull, len(inds))
        rr, ri, gr, gi = o0r.copy(), o0i.copy(), o0r.copy(), o0i.copy()
        ut.convolve_F_general(PQ, F, w[:len(inds)].copy(), rr, ri, n1, n3, n, mu1, inds)
        mine.convolve_F_general(PQ, F, w[:len(inds)].copy(), gr, gi, n1, n3, n, mu1, inds)
        assert close(gr - o0r, rr - o0r, 1e-13) and close(gi - o0i, ri - o0i, 1e-13)


@pytest.mark.gpu
@pytest.mark.parametrize("n1,n3,n", [(1, 2, 1), (2, 2, 2)])
def test_tau_general_many_radii(n1, n3, n):
    """tau_sum_general and convolve_F_general with more than 32 radial samples (the kernels' chunked
    r' path: N_r 37, a 35-sample subset with a zero weight for the convolution) against the compiled
    reference: 1e-12 relative for the sum, 1e-13 of the largest magnitude for the convolutions."""
    from polyspec_b200 import pixel as P
    T, _ = _ref()
    if T is None:
        pytest.skip("oracle/_ref is not built")
    nr = 37
    rng, Ls, F, w, args, nfull = _general_case(nr, max(n, 2), 7 + 100 * n1 + 10 * n3 + n, lmax_L=7, Lmax=5)
    ut, mine = T.tauNL_utils(*args), P.tauNL_utils(*args)

    def cplx(*shape):
        return rng.normal(size=shape) + 1j * rng.normal(size=shape)

    a1, a2 = cplx(2 * n1 + 1, len(Ls), nr), cplx(2 * n3 + 1, len(Ls), nr)
    t_ref, t = ut.tau_sum_general(a1, a2, F, w, n1, n3, n), mine.tau_sum_general(a1, a2, F, w, n1, n3, n)
    assert abs(t - t_ref) <= 1e-12 * max(abs(t_ref), 1e-300), (t, t_ref)
    inds = np.concatenate([np.arange(0, 20), np.arange(22, 37)]).astype(np.int32)
    PQ = cplx(2 * n3 + 1, len(Ls), len(inds))
    wi = w[:len(inds)].copy()
    wi[3] = 0.
    for mu1 in range(-n1, n1 + 1):
        o0r, o0i = cplx(nfull, len(inds)), cplx(nfull, len(inds))
        rr, ri, gr, gi = o0r.copy(), o0i.copy(), o0r.copy(), o0i.copy()
        ut.convolve_F_general(PQ, F, wi, rr, ri, n1, n3, n, mu1, inds)
        mine.convolve_F_general(PQ, F, wi, gr, gi, n1, n3, n, mu1, inds)
        assert close(gr - o0r, rr - o0r, 1e-13) and close(gi - o0i, ri - o0i, 1e-13)
