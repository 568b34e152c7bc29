// Wigner 3j symbols and Gaunt coefficients with one small angular momentum (n, a few
// units) and the other two large, in FP64, for the direction-dependent tauNL
// contractions (the gaunt_symbol of polyspec/cython/tauNL_utils.pyx:1716-1718:
// Gaunt(l1 l2 l3; m1 m2 m3) = sqrt((2l1+1)(2l2+1)(2l3+1)/4pi) (l1 l2 l3; 0 0 0)(l1 l2 l3; m1 m2 m3)).
//
// (l1 l2 n; m1 m2 m3) is written, by the column symmetries, as the Clebsch-Gordan
// coefficient <l1 m1 n m3 | l2 -m2> with the small momentum second, and that by Racah's
// sum.  In the sum every large factorial meets another one whose argument differs by at
// most a few units (the small momentum bounds every difference), so each term is a
// product of short ranges (n!-sized factorials and ratios a!/b! with |a - b| <= 3n): no
// log-gamma of large arguments, no overflow, and the at most 2n + 1 terms keep their
// relative precision (1.5e-13 relative, 1e-15 of the typical magnitude, against exact
// rational evaluation for l up to 3000 and n <= 5).
#pragma once

namespace ps {

// a! / b! for 0 <= a, b, as a product over the range between them
__device__ __forceinline__ double fact_ratio(int a, int b) {
  double r = 1.0;
  if (a >= b) {
    for (int i = b + 1; i <= a; ++i) r *= double(i);
  } else {
    for (int i = a + 1; i <= b; ++i) r /= double(i);
  }
  return r;
}

__device__ __forceinline__ double small_fact(int a) { return fact_ratio(a, 0); }

// <j1 m1 j2 m2 | J M> with j2 small
__device__ inline double cg_small(int j1, int m1, int j2, int m2, int J, int M) {
  if (m1 + m2 != M || abs(m1) > j1 || abs(m2) > j2 || abs(M) > J || J < abs(j1 - j2) || J > j1 + j2) return 0.0;
  const double pre = (2.0 * J + 1.0) * fact_ratio(J + j1 - j2, j1 + j2 + J + 1) * small_fact(J - j1 + j2) *
                     small_fact(j1 + j2 - J) * small_fact(j2 - m2) * small_fact(j2 + m2);
  const int kmin = max(0, max(j2 - J - m1, j1 - J + m2));
  const int kmax = min(j1 + j2 - J, min(j1 - m1, j2 + m2));
  double s = 0.0;
  for (int k = kmin; k <= kmax; ++k) {
    const double big = fact_ratio(j1 - m1, j1 - m1 - k) * sqrt(fact_ratio(J - M, j1 - m1)) *
                       sqrt(fact_ratio(J + M, J - j2 + m1 + k) * fact_ratio(j1 + m1, J - j2 + m1 + k));
    const double small = small_fact(k) * small_fact(j1 + j2 - J - k) * small_fact(j2 + m2 - k) *
                         small_fact(J - j1 - m2 + k);
    s += ((k & 1) ? -big : big) / small;
  }
  return sqrt(pre) * s;
}

// (l1 l2 n; m1 m2 m3) with n small: (-1)^(l1+l2+n) (l1 n l2; m1 m3 m2)
//   = (-1)^(l1+l2+n) (-1)^(l1-n-m2) <l1 m1 n m3 | l2 -m2> / sqrt(2 l2 + 1)
__device__ inline double threej_small(int l1, int l2, int n, int m1, int m2, int m3) {
  if (m1 + m2 + m3 != 0 || l1 < 0 || l2 < 0 || n < 0) return 0.0;
  const int e = (l1 + l2 + n) + (l1 - n - m2);
  const double c = cg_small(l1, m1, n, m3, l2, -m2) / sqrt(2.0 * l2 + 1.0);
  return (e & 1) ? -c : c;
}

__device__ inline double gaunt_small(int l1, int l2, int n, int m1, int m2, int m3) {
  const double t0 = threej_small(l1, l2, n, 0, 0, 0);
  if (t0 == 0.0) return 0.0;
  return threej_small(l1, l2, n, m1, m2, m3) * t0 *
         sqrt((2.0 * l1 + 1.0) * (2.0 * l2 + 1.0) * (2.0 * n + 1.0) / (4.0 * M_PI));
}

}  // namespace ps
