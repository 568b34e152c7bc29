"""ORACLE shim (test infrastructure only): stand-in for pywigxjpf, which the
reference uses for the Wigner 3j symbols of its ideal bispectrum Fisher matrix
(polyspec/bspec_bin.py:122-124) and is not installed here.

wig3jj(2 j1, 2 j2, 2 j3, 2 m1, 2 m2, 2 m3) evaluates the 3j symbol of integer
angular momenta exactly by Racah's formula (rational arithmetic on Python
integers), with the square root taken at 40 digits by mpmath: the value is the
correctly rounded double, as pywigxjpf's exact prime-factor evaluation gives.
wig6jj(2 j1, ..., 2 j6) evaluates the 6j symbol of integer angular momenta the same
way, by Racah's single sum (the reference's tauNL-odd decomposition uses it).
"""
from fractions import Fraction
from functools import lru_cache
from math import factorial

import mpmath


def wig_table_init(*a, **k):
    pass


def wig_temp_init(*a, **k):
    pass


@lru_cache(maxsize=None)
def _three_j(j1, j2, j3, m1, m2, m3):
    if m1 + m2 + m3 != 0 or j3 < abs(j1 - j2) or j3 > j1 + j2:
        return 0.0
    if abs(m1) > j1 or abs(m2) > j2 or abs(m3) > j3:
        return 0.0
    f = factorial
    pref = Fraction(f(j1 + j2 - j3) * f(j1 - j2 + j3) * f(-j1 + j2 + j3), f(j1 + j2 + j3 + 1))
    pref *= f(j1 + m1) * f(j1 - m1) * f(j2 + m2) * f(j2 - m2) * f(j3 + m3) * f(j3 - m3)
    kmin = max(0, j2 - j3 - m1, j1 - j3 + m2)
    kmax = min(j1 + j2 - j3, j1 - m1, j2 + m2)
    s = Fraction(0)
    for k in range(kmin, kmax + 1):
        s += Fraction((-1) ** k, f(k) * f(j3 - j2 + k + m1) * f(j3 - j1 + k - m2) * f(j1 + j2 - j3 - k) *
                      f(j1 - k - m1) * f(j2 - k + m2))
    if s == 0:
        return 0.0
    sign = (-1) ** ((j1 - j2 - m3) % 2) * (1 if s > 0 else -1)
    sq = pref * s * s
    with mpmath.workdps(40):
        return sign * float(mpmath.sqrt(mpmath.mpf(sq.numerator) / sq.denominator))


def wig3jj(tj1, tj2, tj3, tm1, tm2, tm3):
    args = (tj1, tj2, tj3, tm1, tm2, tm3)
    if any(a % 2 for a in args):
        raise NotImplementedError("half-integer angular momenta are outside the oracle's scope")
    return _three_j(*(a // 2 for a in args))


def _delta(a, b, c):
    f = factorial
    return Fraction(f(a + b - c) * f(a - b + c) * f(-a + b + c), f(a + b + c + 1))


@lru_cache(maxsize=None)
def _six_j(j1, j2, j3, j4, j5, j6):
    triads = ((j1, j2, j3), (j1, j5, j6), (j4, j2, j6), (j4, j5, j3))
    if any(c < abs(a - b) or c > a + b for a, b, c in triads):
        return 0.0
    f = factorial
    pref = Fraction(1)
    for a, b, c in triads:
        pref *= _delta(a, b, c)
    A = [a + b + c for a, b, c in triads]
    B = (j1 + j2 + j4 + j5, j2 + j3 + j5 + j6, j3 + j1 + j6 + j4)
    s = Fraction(0)
    for t in range(max(A), min(B) + 1):
        den = 1
        for x in [t - a for a in A] + [b - t for b in B]:
            den *= f(x)
        s += Fraction((-1) ** t * f(t + 1), den)
    if s == 0:
        return 0.0
    sq = pref * s * s
    with mpmath.workdps(40):
        return (1 if s > 0 else -1) * float(mpmath.sqrt(mpmath.mpf(sq.numerator) / sq.denominator))


def wig6jj(*args):
    if any(a % 2 for a in args):
        raise NotImplementedError("half-integer angular momenta are outside the oracle's scope")
    return _six_j(*(a // 2 for a in args))
