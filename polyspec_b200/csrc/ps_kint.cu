// k-space radial integrals of the TSpecTemplate set-up (polyspec/cython/
// k_integrals.pyx), FP64.
//
//  * ps_kint_bessel_table: j_l(x) for l in [lmin, lmax] on a grid of x
//    (k_integrals.pyx:28-71): x = 0 gives (1, 0, 0, ...); x > 18000 + lmax the
//    large-x limit sin(x - l pi/2)/x; otherwise j_l for l up to the largest l whose
//    small-x limit (e x/(2l+1))^(l+1/2)/sqrt(4x(l+1/2)) exceeds 1e-150 (zeros above).
//    The values come from the three-term recurrence j_{l+1} = (2l+1)/x j_l - j_{l-1}:
//    upward from j_0 = sin x / x, j_1 = sin x / x^2 - cos x / x where it is stable
//    (top l below x), otherwise downward (Miller's method) from well above the top l,
//    normalised by the sum rule Sum_l (2l+1) j_l^2 = 1 with the sign of j_0 (or j_1
//    where sin x is tiny); two passes, rescaling by 2^-400 to stay in range.  One
//    thread per x, writes coalesced over x (table [l][x]).
//  * ps_kint_radial: out[l][X][r] += (-1)^l Sum_k (k_i - k_{i-1}) (f_{i-1} + f_i),
//    f_i = kprod_i T_l^X(k_i) j_{l+n}(k_i r) with j interpolated linearly from the
//    table at x = k r (the interval found by bisection: the largest grid point below
//    k r, as numpy's searchsorted(...) - 1 in the reference) -- q_integral
//    (:312-353, kprod = k^2/pi), p_integral (:262-310, kprod = k^2 P_zeta(k)/pi) and
//    r_integral (:355-396, kprod = k^2 P_zeta^(3/4)/pi); with a per-sample kprod[r][k]
//    the (r, tau) integrals a (:127-170), b (:172-215, with j_l' = (l j_{l-1} -
//    (l+1) j_{l+1})/(2l+1) of the interpolated values, as compute_jl_prime :112-124)
//    and c (:217-260, weighted by sqrt(l(l+1))).  One thread per (l, X, r), k summed
//    in order.
#include "ps_common.cuh"
#include "ps_stats.cuh"

namespace ps {
namespace {

constexpr double KI_SMALL = 1e-150;
constexpr double KI_BIG = 0x1p400;  // |f| <= 2^400 keeps (2l+1) f^2 and its sum finite
constexpr double KI_RESCALE = 0x1p-400;

__device__ __forceinline__ double smallx_limit(int l, double x) {
  return pow(M_E * x / (2.0 * l + 1.0), l + 0.5) / sqrt(4.0 * x * (l + 0.5));
}

__global__ void bessel_table_kernel(const double* __restrict__ xs, int64_t nx, int lmin, int lmax,
                                    double* __restrict__ out) {
  for (int64_t ix = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; ix < nx; ix += int64_t(gridDim.x) * blockDim.x) {
    const double x = xs[ix];
    auto put = [&](int l, double v) {
      if (l >= lmin && l <= lmax) out[int64_t(l - lmin) * nx + ix] = v;
    };
    if (x == 0.0) {
      for (int l = lmin; l <= lmax; ++l) put(l, l == 0 ? 1.0 : 0.0);
      continue;
    }
    if (x > 18000.0 + lmax) {
      for (int l = lmin; l <= lmax; ++l) put(l, sin(x - l * M_PI / 2.0) / x);
      continue;
    }
    // top l computed (the rest are zero)
    int lt = lmax;
    if (!(fabs(smallx_limit(lmax, x)) > KI_SMALL)) {
      lt = 1;
      for (int l = lmax; l > 0; --l) {
        if (fabs(smallx_limit(l, x)) > KI_SMALL) { lt = l; break; }
      }
    }
    for (int l = max(lt + 1, lmin); l <= lmax; ++l) put(l, 0.0);
    double s, c;
    sincos(x, &s, &c);
    const double j0 = s / x, j1 = s / (x * x) - c / x;
    if (double(lt) < x) {
      // upward recurrence (stable below the turning point l ~ x)
      double jm = j0, jc = j1;
      put(0, j0);
      if (lt >= 1) put(1, j1);
      for (int l = 1; l < lt; ++l) {
        const double jn = (2.0 * l + 1.0) / x * jc - jm;
        jm = jc;
        jc = jn;
        put(l + 1, jn);
      }
      continue;
    }
    // downward recurrence from L0 well above max(lt, x)
    const double top = fmax(double(lt), x);
    const int L0 = int(top) + 40 + int(sqrt(40.0 * top));
    // pass 1: normalisation and the number of rescalings
    double fp = 0.0, fc = 1.0, sum = 0.0, f0 = 0.0, f1 = 0.0;
    int nres = 0;
    for (int l = L0; l >= 0; --l) {
      sum += (2.0 * l + 1.0) * fc * fc;
      if (l == 1) f1 = fc;
      if (l == 0) { f0 = fc; break; }
      const double fn = (2.0 * l + 1.0) / x * fc - fp;
      fp = fc;
      fc = fn;
      if (fabs(fc) > KI_BIG) {
        fc *= KI_RESCALE;
        fp *= KI_RESCALE;
        sum *= KI_RESCALE * KI_RESCALE;
        ++nres;
      }
    }
    // the sign from j_0, or from j_1 near a zero of j_0 (only signs are compared, so the
    // scale f1 was recorded in does not matter)
    double sign;
    if (fabs(j0) >= fabs(j1)) sign = (f0 >= 0.0) == (j0 >= 0.0) ? 1.0 : -1.0;
    else sign = (f1 >= 0.0) == (j1 >= 0.0) ? 1.0 : -1.0;
    const double inv = sign / sqrt(sum);
    // pass 2: the same recurrence, writing normalised values
    fp = 0.0;
    fc = 1.0;
    int done = 0;
    for (int l = L0; l >= 0; --l) {
      if (l <= lt) {
        double v = fc * inv;
        for (int k = done; k < nres; ++k) v *= KI_RESCALE;
        put(l, v);
      }
      if (l == 0) break;
      const double fn = (2.0 * l + 1.0) / x * fc - fp;
      fp = fc;
      fc = fn;
      if (fabs(fc) > KI_BIG) {
        fc *= KI_RESCALE;
        fp *= KI_RESCALE;
        ++done;
      }
    }
  }
}

__global__ void kint_radial_kernel(const double* __restrict__ table, const double* __restrict__ xs, int64_t nx,
                                   int tab_lmin, int tab_nl, const double* __restrict__ k_arr, int nk,
                                   const double* __restrict__ kprod, int kstride, const double* __restrict__ T,
                                   int npol, int nl_T, const double* __restrict__ r_arr, int nr, int lmin, int lmax,
                                   int nshift, int deriv, int lweight, int npol_out, double* __restrict__ out) {
  const int64_t total = int64_t(lmax - lmin + 1) * npol * nr;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total; t += int64_t(gridDim.x) * blockDim.x) {
    const int ir = int(t % nr);
    const int X = int((t / nr) % npol);
    const int l = lmin + int(t / (int64_t(nr) * npol));
    const int row = l + nshift - tab_lmin;
    if (row < deriv || row + deriv >= tab_nl || l >= nl_T) continue;
    const double r = r_arr[ir];
    const double* jl = table + int64_t(row) * nx;
    const double* jm = jl - nx;  // rows l - 1 and l + 1 (used for j_l')
    const double* jp = jl + nx;
    const double* Tl = T + (int64_t(X) * nl_T + l) * nk;
    const double* kp = kprod + int64_t(kstride) * ir;
    double pref = (l & 1) ? -1.0 : 1.0;
    if (lweight) pref *= sqrt(double(l) * (l + 1.0));
    double acc = 0.0, flow = 0.0;
    for (int ik = 0; ik < nk; ++ik) {
      const double kr = k_arr[ik] * r;
      // largest i with xs[i] < kr (kr > xs[0] = 0 and below the last point)
      int64_t lo = 0, hi = nx - 1;
      while (hi - lo > 1) {
        const int64_t mid = (lo + hi) >> 1;
        if (xs[mid] < kr) lo = mid;
        else hi = mid;
      }
      const double dx = xs[lo + 1] - xs[lo];
      const double xp = (xs[lo + 1] - kr) / dx, xm = (kr - xs[lo]) / dx;
      double j;
      if (deriv) {  // j_l' = (l j_{l-1} - (l+1) j_{l+1}) / (2l+1) of the interpolated values
        const double a = jm[lo] * xp + jm[lo + 1] * xm, b = jp[lo] * xp + jp[lo + 1] * xm;
        j = (l * a - (l + 1.0) * b) / (2.0 * l + 1.0);
      } else {
        j = jl[lo] * xp + jl[lo + 1] * xm;
      }
      const double f = kp[ik] * Tl[ik] * j;
      if (ik > 0) acc += pref * (k_arr[ik] - k_arr[ik - 1]) * (flow + f);
      flow = f;
    }
    out[(int64_t(l) * npol_out + X) * nr + ir] += acc;
  }
}

}  // namespace
}  // namespace ps

using namespace ps;

extern "C" int ps_kint_bessel_table(const double* x, int64_t nx, int lmin, int lmax, double* out,
                                    cudaStream_t stream) {
  if (!x || !out || nx <= 0 || lmin < 0 || lmax < lmin) return PS_ERR_INVALID;
  StatScope sc(PS_K_VECTOR, 0.0, 8.0 * double(nx) * (lmax - lmin + 1), stream);
  int64_t g = (nx + 127) / 128;
  if (g > 65535) g = 65535;
  bessel_table_kernel<<<int(g), 128, 0, stream>>>(x, nx, lmin, lmax, out);
  PS_LAUNCH_CHECK();
  return PS_OK;
}

extern "C" int ps_kint_radial(const double* table, const double* x, int64_t nx, int tab_lmin, int tab_nl,
                              const double* k_arr, int nk, const double* kprod, int kstride, const double* T,
                              int npol, int nl_T, const double* r_arr, int nr, int lmin, int lmax, int nshift,
                              int deriv, int lweight, int npol_out, double* out, cudaStream_t stream) {
  if (!table || !x || !k_arr || !kprod || !T || !r_arr || !out || nx < 2 || tab_nl <= 0 || nk <= 0 || npol <= 0 ||
      nr <= 0 || lmin < 0 || lmax < lmin || npol_out < npol || nl_T <= 0 || (kstride != 0 && kstride != nk) ||
      deriv < 0 || deriv > 1)
    return PS_ERR_INVALID;
  const int64_t total = int64_t(lmax - lmin + 1) * npol * nr;
  StatScope sc(PS_K_VECTOR, 0.0, 8.0 * double(total) * nk, stream);
  int64_t g = (total + 127) / 128;
  if (g > 65535) g = 65535;
  kint_radial_kernel<<<int(g), 128, 0, stream>>>(table, x, nx, tab_lmin, tab_nl, k_arr, nk, kprod, kstride, T,
                                                 npol, nl_T, r_arr, nr, lmin, lmax, nshift, deriv, lweight,
                                                 npol_out, out);
  PS_LAUNCH_CHECK();
  return PS_OK;
}
