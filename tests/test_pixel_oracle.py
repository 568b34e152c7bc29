"""The pixel-product oracle against the reference's own Cython kernels,
compiled from its sources into oracle/_ref (CPU; skipped where the compiled
reference is absent)."""
import os
import sys

import numpy as np
import pytest

import pixel_cases as C

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
from oracle import pixel as O  # noqa: E402


def _ref():
    d = os.path.join(ROOT, "oracle", "_ref")
    if d not in sys.path:
        sys.path.insert(0, d)
    try:
        import tauNL_utils as T
        import ideal_fisher as F
    except ImportError:
        pytest.skip("compiled reference kernels not built (oracle/build_ref.sh)")
    return T, F


def close(a, b, tol):
    a, b = np.asarray(a), np.asarray(b)
    return np.max(np.abs(a - b)) <= tol * max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("op", sorted(C.PRODUCTS))
def test_products_match_reference(op):
    T, F = _ref()
    kinds, fac = C.PRODUCTS[op]
    xs = C.maps(kinds, (3, 1001), seed=sum(map(ord, op)))
    extra = () if fac is None else (fac,)
    if op in C.TAUNL_PRODUCTS:
        ref = getattr(T.tauNL_utils(*C.taunl_args(3, 8)), op)(*xs)
    else:
        ref = getattr(F, op)(*xs, *extra, 2)
    assert close(getattr(O, op)(*xs, *extra), ref, 1e-14)


@pytest.mark.parametrize("kind", sorted(C.SUMS))
def test_radial_sums_match_reference(kind):
    T, _ = _ref()
    kinds, has_tau = C.SUMS[kind]
    nr, npix = 5, 3001
    xs = C.maps(kinds, (nr, npix), seed=17)
    rng = np.random.default_rng(3)
    w, tau = rng.normal(size=nr), rng.uniform(0.5, 2.0, size=nr)
    args = (w, tau) if has_tau else (w,)
    ref = getattr(T.tauNL_utils(*C.taunl_args(nr, 8)), kind)(*args, *xs)
    assert abs(getattr(O, kind)(*args, *xs) - ref) <= 1e-11 * abs(ref)


@pytest.mark.parametrize("npol", [1, 3])
def test_lens_phi_matches_reference(npol):
    _, F = _ref()
    U, V, U2, V2 = C.maps("cccc", (npol, 777), seed=npol)
    assert close(O.lens_phi_sum(U, V), F.lens_phi_sum(U, V, 2), 1e-14)
    assert close(O.lens_phi_sum_sym(U, U2, V, V2), F.lens_phi_sum_sym(U, U2, V, V2, 2), 1e-14)


@pytest.mark.parametrize("npol", [1, 2, 3])
def test_harmonic_weightings_match_reference(npol):
    T, _ = _ref()
    lmax, nr = 12, 7
    l, m = C.lm_setup(lmax)
    rng = np.random.default_rng(npol)
    flX = rng.normal(size=(lmax + 1, npol, nr))
    h = rng.normal(size=(npol, len(l))) + 1j * rng.normal(size=(npol, len(l)))
    t = T.tauNL_utils(*C.taunl_args(nr, lmax))
    assert close(O.apply_fl_weights(l, flX, h, 0.3), t.apply_fl_weights(flX, h, 0.3), 1e-14)
    lm_map = rng.normal(size=(nr, len(l))) + 1j * rng.normal(size=(nr, len(l)))
    w = rng.normal(size=nr)
    assert close(O.radial_sum(l, lm_map, w, flX), t.radial_sum(lm_map, w, flX), 1e-13)
    lm2 = rng.normal(size=(2, nr, len(l))) + 1j * rng.normal(size=(2, nr, len(l)))
    assert close(O.radial_sum_spin1(l, lm2, w, flX), t.radial_sum_spin1(lm2, w, flX), 1e-13)


@pytest.mark.parametrize("sym", [False, True])
def test_outer_product_matches_reference(sym):
    _, F = _ref()
    rng = np.random.default_rng(5)
    Qa = rng.normal(size=(4, 6, 500)) + 1j * rng.normal(size=(4, 6, 500))
    Qb = Qa if sym else rng.normal(size=(4, 9, 500)) + 1j * rng.normal(size=(4, 9, 500))
    assert close(O.outer_product(Qa, Qb, sym), F.outer_product(Qa, Qb, 2, sym), 1e-12)
