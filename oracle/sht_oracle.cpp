// ORACLE -- test infrastructure only.  Nothing in the product path may link,
// load or call this file; only tests/, __graft_entry__.smoke() and the
// cpu_baseline / --impl reference legs of bench.py use it, as the checker.
//
// FP64 CPU restatement of the HEALPix spin-0 / spin-s spherical harmonic
// transforms that the reference reaches through the third-party ducc0 package:
//
//   ducc0.sht.synthesis          polyspec/base.py:172-176, 225, 230-231, 282
//   ducc0.sht.adjoint_synthesis  polyspec/base.py:147-151, 193, 206, 253
//   ducc0.healpix.Healpix_Base(nside,"RING").sht_info()   polyspec/base.py:72-73
//
// ducc0 is not vendored by the reference and its version is not pinned
// (README.md:69-75 lists "ducc0" with no version); it is absent from this
// container.  What is restated here is the published algorithm:
//   * HEALPix RING geometry: Gorski et al. 2005, ApJ 622:759, section 4.
//   * normalised associated-Legendre / spin-weighted harmonic recurrences with
//     scaled seeds: Reinecke & Seljebotn 2013, A&A 554, A112 (libsharp).
//   * spin-weighted harmonics sY_lm in the Goldberg et al. (1967) convention,
//     which is the HEALPix one: sY_lm = sqrt((l-s)!/(l+s)!) eth^s Y_lm with
//     eth f = -(sin th)^s (d_th + i/sin th d_ph)(sin th)^-s f.
//   * HEALPix spin conventions (polyspec/base.py:247, 255-256, 276, 285-286):
//     +s a_lm = -(G + iC),  -s a_lm = -(-1)^s (G - iC),
//     Q + iU = sum +s a_lm +sY_lm,  Q - iU = sum -s a_lm -sY_lm.
//   * adjoint_synthesis = exact adjoint of synthesis under the m-weighted alm
//     inner product Re sum_{l,m>=0} (1+[m>0]) a* b  (the CG dot product of
//     polyspec/weighting.py:255): a_lm = sum_p map(p) Y*_lm(p).
// Ring transforms are an exact DFT per ring with HEALPix m-aliasing; two
// evaluation modes exist: a direct O(N^2) DFT (the definition) and an FFT
// (radix-2 + Bluestein chirp-z), cross-checked against each other in tests.

#include <cmath>
#include <complex>
#include <vector>
#include <algorithm>
#include <cstring>
#include <cstdint>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef std::complex<double> cplx;

namespace {

struct Ring {
  double z;      // cos(theta)
  double omz;    // 1 - z, accurate near the north pole
  double opz;    // 1 + z, accurate near the south pole
  double sth;    // sin(theta)
  double phi0;   // longitude of the first pixel centre
  int64_t nphi;  // pixels in the ring
  int64_t start; // index of the first pixel
};

// HEALPix RING scheme: rings i = 1..4 nside-1 from the north pole.
std::vector<Ring> healpix_rings(int nside) {
  const int64_t ns = nside, npix = 12 * ns * ns;
  const int R = 4 * nside - 1;
  std::vector<Ring> out(R);
  for (int ir = 0; ir < R; ++ir) {
    const int64_t i = ir + 1;
    const bool north = i <= 2 * ns;
    const int64_t ii = north ? i : 4 * ns - i;  // ring number counted from the nearer pole
    Ring g;
    if (ii < ns) {
      const double t = double(ii * ii) / (3.0 * double(ns * ns));  // 1 - |z|
      g.z = north ? 1.0 - t : t - 1.0;
      g.omz = north ? t : 2.0 - t;
      g.opz = north ? 2.0 - t : t;
      g.sth = std::sqrt(t * (2.0 - t));
      g.nphi = 4 * ii;
      g.phi0 = M_PI / (4.0 * double(ii));
      g.start = north ? 2 * ii * (ii - 1) : npix - 2 * ii * (ii + 1);
    } else {
      const double z = double(2 * ns - i) * 2.0 / (3.0 * double(ns));
      g.z = z;
      g.omz = 1.0 - z;
      g.opz = 1.0 + z;
      g.sth = std::sqrt(g.omz * g.opz);
      g.nphi = 4 * ns;
      g.phi0 = ((i - ns) % 2 == 0) ? M_PI / (4.0 * double(ns)) : 0.0;
      g.start = 2 * ns * (ns - 1) + (i - ns) * 4 * ns;
    }
    out[ir] = g;
  }
  return out;
}

// ---------------------------------------------------------------- scaled reals
// value = v * 2^e with v in [0.5, 1) (or 0)
struct Scaled { double v; int64_t e; };

Scaled snorm(double x) { int e; double v = std::frexp(x, &e); return {v, e}; }
Scaled smul(Scaled a, Scaled b) { Scaled r = snorm(a.v * b.v); r.e += a.e + b.e; return r; }
Scaled spow(double x, int n) {  // x > 0, n >= 0, binary exponentiation
  Scaled r{0.5, 1}, b = snorm(x);
  while (n) { if (n & 1) r = smul(r, b); b = smul(b, b); n >>= 1; }
  return r;
}

// Large-exponent bookkeeping of the recurrence: true value = v * FBIG^k, k <= 0.
const int SCALE_BITS = 800;
const double FBIG = std::ldexp(1.0, SCALE_BITS);
const double FSMALL = std::ldexp(1.0, -SCALE_BITS);
const double FTHRESH = std::ldexp(1.0, SCALE_BITS / 2);

// split a Scaled into (v', k) with v' * FBIG^k == value and, when k < 0,
// |v'| <= FTHRESH; values above 2^-(SCALE_BITS/2) get k = 0.
inline void to_kscale(Scaled s, double& v, int& k) {
  if (s.v == 0.0) { v = 0.0; k = 0; return; }
  int64_t e = s.e;
  k = 0;
  if (e <= -SCALE_BITS / 2) {
    int64_t steps = (-SCALE_BITS / 2 - e) / SCALE_BITS + 1;  // e + steps*SCALE_BITS in (-SCALE_BITS/2, SCALE_BITS/2]
    e += steps * SCALE_BITS;
    k = steps > 1000000 ? -1000000 : -(int)steps;
  }
  v = std::ldexp(s.v, (int)e);
}

// log2 of binomial C(n, k) as a Scaled value, computed by products
Scaled sbinom(int n, int k) {
  Scaled r{0.5, 1};
  for (int j = 1; j <= k; ++j) r = smul(r, snorm(double(n - k + j) / double(j)));
  return r;
}

// ---------------------------------------------------------------- Legendre
// Per-m coefficient tables.
struct Coef0 { std::vector<double> a, b; };  // spin 0: lam_l = a_l (x lam_{l-1}) - b_l lam_{l-2}

// spin-0: lam_{l} = a_l * x * lam_{l-1} - b_l * lam_{l-2},
//   a_l = sqrt((4l^2-1)/(l^2-m^2)), b_l = a_l / a_{l-1}
Coef0 coef_spin0(int m, int lmax) {
  Coef0 c; c.a.assign(lmax + 2, 0.0); c.b.assign(lmax + 2, 0.0);
  auto al = [&](int l) { return std::sqrt((4.0 * l * l - 1.0) / (double(l) * l - double(m) * m)); };
  for (int l = m + 1; l <= lmax; ++l) {
    c.a[l] = al(l);
    c.b[l] = (l >= m + 2) ? c.a[l] / al(l - 1) : 0.0;
  }
  return c;
}

// spin s > 0: for f = +s lam and g = -s lam
//   f_{l+1} = (A_l x + D_l) f_l - C_l f_{l-1},  g_{l+1} = (A_l x - D_l) g_l - C_l g_{l-1}
//   A_l = sqrt((2l+3)(2l+1)) (l+1) / rho_{l+1}
//   D_l = sqrt((2l+3)(2l+1)) m s / (l rho_{l+1})
//   C_l = sqrt((2l+3)/(2l-1)) (l+1) rho_l / (l rho_{l+1}),  rho_l = sqrt((l^2-m^2)(l^2-s^2))
struct CoefS { std::vector<double> A, D, C; };
CoefS coef_spin(int m, int s, int lmax) {
  CoefS c; c.A.assign(lmax + 2, 0.0); c.D.assign(lmax + 2, 0.0); c.C.assign(lmax + 2, 0.0);
  auto rho = [&](int l) {
    double t1 = double(l) * l - double(m) * m, t2 = double(l) * l - double(s) * s;
    return std::sqrt(std::max(t1, 0.0) * std::max(t2, 0.0));
  };
  const int lmin = std::max(m, s);
  for (int l = lmin; l < lmax; ++l) {
    double r1 = rho(l + 1), q = std::sqrt((2.0 * l + 3.0) * (2.0 * l + 1.0));
    c.A[l] = q * (l + 1.0) / r1;
    c.D[l] = q * double(m) * double(s) / (double(l) * r1);
    c.C[l] = std::sqrt((2.0 * l + 3.0) / (2.0 * l - 1.0)) * (l + 1.0) * rho(l) / (double(l) * r1);
  }
  return c;
}

// Evaluate lam_lm(theta), l = m..lmax (spin 0) into out[l-m]; entries below the
// FP64 range (scaled exponent k < 0) are written as 0.
void legendre_spin0(int m, int lmax, const Coef0& c, const Ring& g, const std::vector<double>& mnorm, double* out) {
  // lam_mm = (-1)^m mnorm[m] sin^m th
  Scaled st = spow(g.sth, m);
  Scaled s0 = smul(st, snorm(mnorm[m]));
  double v; int k; to_kscale(s0, v, k);
  if (m & 1) v = -v;
  double prev = 0.0, cur = v;
  const double x = g.z;
  for (int l = m; l <= lmax; ++l) {
    out[l - m] = (k == 0) ? cur : 0.0;
    if (l == lmax) break;
    double nxt = c.a[l + 1] * x * cur - c.b[l + 1] * prev;
    prev = cur; cur = nxt;
    if (k < 0 && std::fabs(cur) > FTHRESH) { cur *= FSMALL; prev *= FSMALL; ++k; }
  }
}

// Evaluate F+ = (+s lam + -s lam)/2 and F- = (+s lam - -s lam)/2 for l = lmin..lmax
// (entries l < lmin are 0).  Output index is l - m.
// sqrt((2 lmin+1)/(4 pi) C(2 lmin, lmin + min(m,s)... )) : the l = lmin seed normalisation, per m
Scaled spin_seed_norm(int m, int s) {
  Scaled nrm = (m >= s) ? smul(sbinom(2 * m, m + s), snorm((2.0 * m + 1.0) / (4.0 * M_PI)))
                        : smul(sbinom(2 * s, s + m), snorm((2.0 * s + 1.0) / (4.0 * M_PI)));
  double v = nrm.v; int64_t e = nrm.e;
  if (e & 1) { v *= 2.0; e -= 1; }
  Scaled r = snorm(std::sqrt(v)); r.e += e / 2;
  return r;
}

void legendre_spin(int m, int s, int lmax, const CoefS& c, const Ring& g, Scaled nrm, double* Fp, double* Fm) {
  const int lmin = std::max(m, s);
  for (int l = m; l < lmin && l <= lmax; ++l) { Fp[l - m] = 0.0; Fm[l - m] = 0.0; }
  if (lmin > lmax) return;
  // sin(th/2), cos(th/2)
  const double sh = std::sqrt(0.5 * g.omz), ch = std::sqrt(0.5 * g.opz);
  // seeds at l = lmin (Goldberg et al. 1967 with one term left in the sum):
  //   m >= s: +s lam = (-1)^m N sin^{m+s}(th/2) cos^{m-s}(th/2), -s lam = (-1)^m N sin^{m-s} cos^{m+s}
  //   m <  s: +s lam = (-1)^m N sin^{s+m} cos^{s-m},             -s lam = (-1)^s N sin^{s-m} cos^{s+m}
  Scaled pf, pg;
  double sgn_f, sgn_g;
  if (m >= s) {
    pf = smul(spow(sh, m + s), spow(ch, m - s));
    pg = smul(spow(sh, m - s), spow(ch, m + s));
    sgn_f = (m & 1) ? -1.0 : 1.0;
    sgn_g = sgn_f;
  } else {
    pf = smul(spow(sh, s + m), spow(ch, s - m));
    pg = smul(spow(sh, s - m), spow(ch, s + m));
    sgn_f = (m & 1) ? -1.0 : 1.0;
    sgn_g = (s & 1) ? -1.0 : 1.0;
  }
  Scaled sf = smul(nrm, pf), sg = smul(nrm, pg);
  // common scale from the larger one
  Scaled big = (sf.e >= sg.e) ? sf : sg;
  double vb; int k; to_kscale(big, vb, k);
  const int64_t shift = int64_t(k) * SCALE_BITS;  // value = v * 2^shift
  double f = std::ldexp(sf.v, (int)std::max<int64_t>(sf.e - shift, -2000)) * sgn_f;
  double gg = std::ldexp(sg.v, (int)std::max<int64_t>(sg.e - shift, -2000)) * sgn_g;
  double fprev = 0.0, gprev = 0.0;
  const double x = g.z;
  for (int l = lmin; l <= lmax; ++l) {
    if (k == 0) { Fp[l - m] = 0.5 * (f + gg); Fm[l - m] = 0.5 * (f - gg); }
    else { Fp[l - m] = 0.0; Fm[l - m] = 0.0; }
    if (l == lmax) break;
    double ax = c.A[l] * x;
    double fn = (ax + c.D[l]) * f - c.C[l] * fprev;
    double gn = (ax - c.D[l]) * gg - c.C[l] * gprev;
    fprev = f; f = fn; gprev = gg; gg = gn;
    if (k < 0 && std::max(std::fabs(f), std::fabs(gg)) > FTHRESH) {
      f *= FSMALL; fprev *= FSMALL; gg *= FSMALL; gprev *= FSMALL; ++k;
    }
  }
}

std::vector<double> spin0_mnorm(int mmax) {
  // sqrt((2m+1)/(4 pi) * prod_{k=1..m} (2k-1)/(2k))
  std::vector<double> out(mmax + 1);
  double p = 1.0;
  for (int m = 0; m <= mmax; ++m) {
    if (m > 0) p *= (2.0 * m - 1.0) / (2.0 * m);
    out[m] = std::sqrt((2.0 * m + 1.0) / (4.0 * M_PI) * p);
  }
  return out;
}

// ---------------------------------------------------------------- ring DFT
void fft_pow2(cplx* a, int n, int sign) {  // in place, radix-2 DIT, e^{sign 2 pi i jk/n}
  for (int i = 1, j = 0; i < n; ++i) {
    int bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) std::swap(a[i], a[j]);
  }
  for (int len = 2; len <= n; len <<= 1) {
    for (int i = 0; i < n; i += len) {
      for (int j = 0; j < len / 2; ++j) {
        double ang = sign * 2.0 * M_PI * j / len;
        cplx w(std::cos(ang), std::sin(ang));
        cplx u = a[i + j], v = a[i + j + len / 2] * w;
        a[i + j] = u + v;
        a[i + j + len / 2] = u - v;
      }
    }
  }
}

// X_k = sum_j x_j e^{sign 2 pi i jk/n}, any n
void dft_any(const cplx* x, cplx* X, int n, int sign, bool direct) {
  if (direct || n <= 8) {
    for (int k = 0; k < n; ++k) {
      cplx s = 0.0;
      for (int j = 0; j < n; ++j) {
        int64_t jk = (int64_t(j) * k) % n;
        double ang = sign * 2.0 * M_PI * double(jk) / n;
        s += x[j] * cplx(std::cos(ang), std::sin(ang));
      }
      X[k] = s;
    }
    return;
  }
  if ((n & (n - 1)) == 0) {
    std::vector<cplx> a(x, x + n);
    fft_pow2(a.data(), n, sign);
    std::copy(a.begin(), a.end(), X);
    return;
  }
  // Bluestein: jk = (j^2 + k^2 - (k-j)^2)/2
  int M = 1; while (M < 2 * n - 1) M <<= 1;
  std::vector<cplx> w(n), a(M, 0.0), b(M, 0.0);
  for (int j = 0; j < n; ++j) {
    int64_t q = (int64_t(j) * j) % (2 * n);
    double ang = sign * M_PI * double(q) / n;
    w[j] = cplx(std::cos(ang), std::sin(ang));
  }
  for (int j = 0; j < n; ++j) a[j] = x[j] * w[j];
  b[0] = std::conj(w[0]);
  for (int j = 1; j < n; ++j) { b[j] = std::conj(w[j]); b[M - j] = std::conj(w[j]); }
  fft_pow2(a.data(), M, -1);
  fft_pow2(b.data(), M, -1);
  for (int i = 0; i < M; ++i) a[i] *= b[i];
  fft_pow2(a.data(), M, +1);
  for (int k = 0; k < n; ++k) X[k] = w[k] * a[k] / double(M);
}

// map_j = sum_{|m|<=mmax} F_m e^{i m (phi0 + 2 pi j/n)}, F_{-m} = conj(F_m)
void ring_synth(const cplx* F, int mmax, const Ring& g, double* out, bool direct) {
  const int n = (int)g.nphi;
  std::vector<cplx> c(n, 0.0), X(n);
  for (int m = 0; m <= mmax; ++m) {
    cplx v = F[m] * std::polar(1.0, m * g.phi0);
    c[m % n] += v;
    if (m > 0) c[(n - (m % n)) % n] += std::conj(v);
  }
  dft_any(c.data(), X.data(), n, +1, direct);
  for (int j = 0; j < n; ++j) out[j] = X[j].real();
}

// P_m = sum_j map_j e^{-i m (phi0 + 2 pi j/n)}, m = 0..mmax
void ring_adjoint(const double* in, int mmax, const Ring& g, cplx* P, bool direct) {
  const int n = (int)g.nphi;
  std::vector<cplx> x(n), X(n);
  for (int j = 0; j < n; ++j) x[j] = in[j];
  dft_any(x.data(), X.data(), n, -1, direct);
  for (int m = 0; m <= mmax; ++m) P[m] = X[m % n] * std::polar(1.0, -m * g.phi0);
}

inline int64_t alm_index(int l, int m, int lmax) { return int64_t(m) * (2 * lmax + 1 - m) / 2 + l; }

}  // namespace

extern "C" {

int orc_ring_info(int nside, double* theta, double* phi0, int64_t* nphi, int64_t* ringstart) {
  if (nside < 1) return -1;
  auto r = healpix_rings(nside);
  for (size_t i = 0; i < r.size(); ++i) {
    theta[i] = std::atan2(r[i].sth, r[i].z);
    phi0[i] = r[i].phi0;
    nphi[i] = r[i].nphi;
    ringstart[i] = r[i].start;
  }
  return 0;
}

// Legendre values for tests: out[(l-m)] for one (m, ring); spin 0 -> lam,
// spin > 0 -> F+ in out, F- in out2.
int orc_legendre(int nside, int ring, int lmax, int m, int spin, double* out, double* out2) {
  auto r = healpix_rings(nside);
  if (ring < 0 || ring >= (int)r.size() || m < 0 || m > lmax) return -1;
  if (spin == 0) {
    auto c = coef_spin0(m, lmax);
    auto mn = spin0_mnorm(m);
    legendre_spin0(m, lmax, c, r[ring], mn, out);
  } else {
    auto c = coef_spin(m, spin, lmax);
    legendre_spin(m, spin, lmax, c, r[ring], spin_seed_norm(m, spin), out, out2);
  }
  return 0;
}

// alm: complex128 [nmaps][ncomp][nalm];  map: float64 [nmaps][ncomp][npix]
// ncomp = 1 for spin 0, 2 (G,C -> Q,U) for spin > 0.
int orc_synthesis(int nside, int lmax, int mmax, int spin, int nmaps, const double* alm_ri, double* map,
                  int nthreads, int direct) {
  if (nside < 1 || lmax < 0 || mmax != lmax || spin < 0 || nmaps < 0) return -1;
  const cplx* alm = reinterpret_cast<const cplx*>(alm_ri);
  const auto rings = healpix_rings(nside);
  const int R = (int)rings.size(), Rh = 2 * nside;  // ring pairs (the last is the equator)
  const int64_t npix = 12 * int64_t(nside) * nside;
  const int64_t nalm_full = int64_t(mmax + 1) * (mmax + 2) / 2 + int64_t(mmax + 1) * (lmax - mmax);
  const int ncomp = spin == 0 ? 1 : 2;
  const int nf = nmaps * ncomp;
  if (nthreads <= 0) nthreads = 1;
  std::vector<cplx> phase(size_t(R) * (mmax + 1) * nf);  // [ring][m][f]
  auto mnorm = spin0_mnorm(mmax);
#pragma omp parallel num_threads(nthreads)
  {
    std::vector<double> lam(lmax + 2), lam2(lmax + 2);
#pragma omp for schedule(dynamic, 1)
    for (int m = 0; m <= mmax; ++m) {
      Coef0 c0; CoefS cs; Scaled snrm{0.5, 1};
      if (spin == 0) c0 = coef_spin0(m, lmax);
      else { cs = coef_spin(m, spin, lmax); snrm = spin_seed_norm(m, spin); }
      const int64_t base = alm_index(m, m, lmax);
      for (int rp = 0; rp < Rh; ++rp) {
        const Ring& g = rings[rp];
        const int rs = R - 1 - rp;  // mirror ring (== rp for the equator)
        const bool pair = rs != rp;
        if (spin == 0) {
          legendre_spin0(m, lmax, c0, g, mnorm, lam.data());
          for (int b = 0; b < nmaps; ++b) {
            const cplx* a = alm + int64_t(b) * nalm_full + base;
            cplx s0 = 0.0, s1 = 0.0;
            for (int l = m; l <= lmax; ++l) {
              if ((l + m) & 1) s1 += lam[l - m] * a[l - m]; else s0 += lam[l - m] * a[l - m];
            }
            phase[(size_t(rp) * (mmax + 1) + m) * nf + b] = s0 + s1;
            if (pair) phase[(size_t(rs) * (mmax + 1) + m) * nf + b] = s0 - s1;
          }
        } else {
          legendre_spin(m, spin, lmax, cs, g, snrm, lam.data(), lam2.data());
          for (int b = 0; b < nmaps; ++b) {
            const cplx* G = alm + (int64_t(b) * 2 + 0) * nalm_full + base;
            const cplx* C = alm + (int64_t(b) * 2 + 1) * nalm_full + base;
            cplx GP[2] = {0.0, 0.0}, GM[2] = {0.0, 0.0}, CP[2] = {0.0, 0.0}, CM[2] = {0.0, 0.0};
            for (int l = m; l <= lmax; ++l) {
              const int p = (l + m) & 1;
              const double fp = lam[l - m], fm = lam2[l - m];
              GP[p] += fp * G[l - m]; GM[p] += fm * G[l - m];
              CP[p] += fp * C[l - m]; CM[p] += fm * C[l - m];
            }
            const cplx I(0.0, 1.0);
            for (int side = 0; side < (pair ? 2 : 1); ++side) {
              // north: F+ -> +, F- -> +; south: F+ -> (-1)^p, F- -> -(-1)^p
              cplx gp = side == 0 ? GP[0] + GP[1] : GP[0] - GP[1];
              cplx gm = side == 0 ? GM[0] + GM[1] : -GM[0] + GM[1];
              cplx cp = side == 0 ? CP[0] + CP[1] : CP[0] - CP[1];
              cplx cm = side == 0 ? CM[0] + CM[1] : -CM[0] + CM[1];
              cplx q, u;
              if ((spin & 1) == 0) { q = -(gp + I * cm); u = I * gm - cp; }
              else { q = -(gm + I * cp); u = I * gp - cm; }
              const int rr = side == 0 ? rp : rs;
              phase[(size_t(rr) * (mmax + 1) + m) * nf + 2 * b + 0] = q;
              phase[(size_t(rr) * (mmax + 1) + m) * nf + 2 * b + 1] = u;
            }
          }
        }
      }
    }
#pragma omp for schedule(dynamic, 4)
    for (int ir = 0; ir < R; ++ir) {
      std::vector<cplx> F(mmax + 1);
      for (int f = 0; f < nf; ++f) {
        for (int m = 0; m <= mmax; ++m) F[m] = phase[(size_t(ir) * (mmax + 1) + m) * nf + f];
        ring_synth(F.data(), mmax, rings[ir], map + int64_t(f) * npix + rings[ir].start, direct != 0);
      }
    }
  }
  return 0;
}

int orc_adjoint(int nside, int lmax, int mmax, int spin, int nmaps, const double* map, double* alm_ri,
                int nthreads, int direct) {
  if (nside < 1 || lmax < 0 || mmax != lmax || spin < 0 || nmaps < 0) return -1;
  cplx* alm = reinterpret_cast<cplx*>(alm_ri);
  const auto rings = healpix_rings(nside);
  const int R = (int)rings.size(), Rh = 2 * nside;
  const int64_t npix = 12 * int64_t(nside) * nside;
  const int64_t nalm_full = int64_t(mmax + 1) * (mmax + 2) / 2 + int64_t(mmax + 1) * (lmax - mmax);
  const int ncomp = spin == 0 ? 1 : 2;
  const int nf = nmaps * ncomp;
  if (nthreads <= 0) nthreads = 1;
  std::vector<cplx> phase(size_t(R) * (mmax + 1) * nf);
  auto mnorm = spin0_mnorm(mmax);
#pragma omp parallel num_threads(nthreads)
  {
#pragma omp for schedule(dynamic, 4)
    for (int ir = 0; ir < R; ++ir) {
      std::vector<cplx> P(mmax + 1);
      for (int f = 0; f < nf; ++f) {
        ring_adjoint(map + int64_t(f) * npix + rings[ir].start, mmax, rings[ir], P.data(), direct != 0);
        for (int m = 0; m <= mmax; ++m) phase[(size_t(ir) * (mmax + 1) + m) * nf + f] = P[m];
      }
    }
    std::vector<double> lam(lmax + 2), lam2(lmax + 2);
#pragma omp for schedule(dynamic, 1)
    for (int m = 0; m <= mmax; ++m) {
      Coef0 c0; CoefS cs; Scaled snrm{0.5, 1};
      if (spin == 0) c0 = coef_spin0(m, lmax);
      else { cs = coef_spin(m, spin, lmax); snrm = spin_seed_norm(m, spin); }
      const int64_t base = alm_index(m, m, lmax);
      for (int f = 0; f < nf; ++f)
        for (int l = m; l <= lmax; ++l) alm[int64_t(f) * nalm_full + base + (l - m)] = 0.0;
      for (int rp = 0; rp < Rh; ++rp) {
        const Ring& g = rings[rp];
        const int rs = R - 1 - rp;
        const bool pair = rs != rp;
        auto ph = [&](int ring, int f) { return phase[(size_t(ring) * (mmax + 1) + m) * nf + f]; };
        if (spin == 0) {
          legendre_spin0(m, lmax, c0, g, mnorm, lam.data());
          for (int b = 0; b < nmaps; ++b) {
            const cplx pn = ph(rp, b), ps = pair ? ph(rs, b) : cplx(0.0);
            const cplx pe = pn + ps, po = pn - ps;
            cplx* a = alm + int64_t(b) * nalm_full + base;
            for (int l = m; l <= lmax; ++l) a[l - m] += lam[l - m] * (((l + m) & 1) ? po : pe);
          }
        } else {
          legendre_spin(m, spin, lmax, cs, g, snrm, lam.data(), lam2.data());
          const cplx I(0.0, 1.0);
          for (int b = 0; b < nmaps; ++b) {
            const cplx qn = ph(rp, 2 * b), qs = pair ? ph(rs, 2 * b) : cplx(0.0);
            const cplx un = ph(rp, 2 * b + 1), us = pair ? ph(rs, 2 * b + 1) : cplx(0.0);
            cplx* G = alm + (int64_t(b) * 2 + 0) * nalm_full + base;
            cplx* C = alm + (int64_t(b) * 2 + 1) * nalm_full + base;
            for (int l = m; l <= lmax; ++l) {
              const int p = (l + m) & 1;
              // multiplies F+: north + (-1)^p south; multiplies F-: north - (-1)^p south
              const cplx qp = p ? qn - qs : qn + qs, qm = p ? qn + qs : qn - qs;
              const cplx up = p ? un - us : un + us, um = p ? un + us : un - us;
              const double fp = lam[l - m], fm = lam2[l - m];
              if ((spin & 1) == 0) {
                G[l - m] += -fp * qp - I * fm * um;
                C[l - m] += I * fm * qm - fp * up;
              } else {
                G[l - m] += -fm * qm - I * fp * up;
                C[l - m] += I * fp * qp - fm * um;
              }
            }
          }
        }
      }
    }
  }
  return 0;
}

}  // extern "C"
