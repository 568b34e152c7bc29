// Local-tauNL radial kernels of the TSpecTemplate estimator (FP64).
//
//  * ps_tau_F_integral: F_{L,L+n}(r, r') of polyspec/cython/k_integrals.pyx:453-494
//    (compute_F_integral), the closed form of the k integral of two spherical Bessel
//    functions against the power-law P_zeta:
//      r <= r':  F = A_L 2F1(i1, i2a; i3a; (r/r')^2) (r/r')^L r'^(1-ns)
//      r >  r':  F = B_L 2F1(i1, i2b; i3b; (r'/r)^2) (r'/r)^(L+n) r^(1-ns)
//    with i1 = L + (n-1+ns)/2, i2a/b = (ns-2-/+n)/2, i3a = L + 3/2, i3b = L + n + 3/2
//    and A_L, B_L = 2^(ns-3) pref Gamma(i1) / (Gamma(1-i2a/b) Gamma(i3a/b)) (log-gamma
//    differences).  The reference calls GSL's gsl_sf_hyperg_2F1; here 2F1 is evaluated
//    from its Gauss series, or -- where z is close to 1 and the parameters are small
//    enough that the two terms do not cancel -- from the standard z -> 1 - z connection
//    formula (Abramowitz & Stegun 15.3.6, valid for non-integer c - a - b), and at
//    z = 1 from Gauss's summation theorem.  One thread per (n, L, r, r').  A series that
//    does not converge within its iteration limit sets an error flag.
//  * ps_tau_convolve_F: out[j][lm] = Sum_k F_L(r_j, r_k) w_k X[k][lm] / sqrt(4 pi), F stored
//    [j][k][L] so that a warp's lanes (consecutive lm of one m: consecutive L) read
//    consecutive words (an [L][j][k] layout left the kernel bound by L1 wavefronts)
//    for lm with Lmin <= L <= Lmax (zero elsewhere), the n = n1 = n3 = 0 convolution
//    tauNL_utils.pyx:966-995 (convolve_F_n000), skipping r_k with w_k = 0.  With A
//    given it also returns
//      Sum_{lm, j} m_w(lm) w_j Re(A[j][lm] conj(out[j][lm])),
//    which equals tau_sum_n0 (tauNL_utils.pyx:604-647) of (A, X) since F_L is
//    symmetric for n = 0.  A CTA stages X for a tile of 32 lm and all radial samples in
//    shared memory and computes the tile for every r_j; the dot product reduces per
//    CTA into partials summed in a fixed order by a second kernel.
#include "ps_common.cuh"
#include "ps_stats.cuh"

namespace ps {
namespace {

constexpr int TAU_TILE = 32;      // lm per CTA
constexpr int TAU_JLANES = 8;     // radial lanes per CTA
constexpr int TAU_THREADS = TAU_TILE * TAU_JLANES;
constexpr int HYP_MAXIT = 4000000;

// log|Gamma(x)| and the sign of Gamma(x); *sign = 0 at the poles (x a non-positive integer)
__device__ double lgamma_signed(double x, double* sign) {
  if (x > 0.0) {
    *sign = 1.0;
    return lgamma(x);
  }
  if (x == floor(x)) {
    *sign = 0.0;
    return 0.0;
  }
  *sign = (static_cast<long long>(floor(x)) & 1LL) ? -1.0 : 1.0;
  return lgamma(x);
}

// Gauss series Sum_k (a)_k (b)_k / ((c)_k k!) z^k, stopped once the remaining geometric tail is
// below 1e-17 of the sum; *ok = 0 if that takes more than HYP_MAXIT terms.
__device__ double hyp2f1_series(double a, double b, double c, double z, int* ok) {
  double sum = 1.0, term = 1.0;
  // past k = kmin no factor (b + k), (c + k) changes sign, so the terms keep one sign and their ratio
  // moves monotonically towards z: the tail is bounded by a geometric series of ratio max(|ratio|, |z|)
  const double kmin = fmax(fmax(-b, -c), 0.0) + 2.0;
  for (int k = 0; k < HYP_MAXIT; ++k) {
    const double dk = double(k);
    const double ratio = (a + dk) * (b + dk) / ((c + dk) * (dk + 1.0)) * z;
    term *= ratio;
    sum += term;
    if (term == 0.0) return sum;
    const double rb = fmax(fabs(ratio), fabs(z));
    if (dk > kmin && rb < 1.0 && fabs(term) * rb <= 1e-17 * fabs(sum) * (1.0 - rb)) return sum;
  }
  *ok = 0;
  return sum;
}

__device__ double hyp2f1(double a, double b, double c, double z, int* ok) {
  if (z == 0.0) return 1.0;
  const double s = c - a - b;
  if (z == 1.0) {  // Gauss: Gamma(c) Gamma(c-a-b) / (Gamma(c-a) Gamma(c-b)), for c - a - b > 0
    if (!(s > 0.0)) {
      *ok = 0;
      return 0.0;
    }
    double s1, s2, s3, s4;
    const double lg = lgamma_signed(c, &s1) + lgamma_signed(s, &s2) - lgamma_signed(c - a, &s3) -
                      lgamma_signed(c - b, &s4);
    if (s3 == 0.0 || s4 == 0.0) return 0.0;
    return s1 * s2 * s3 * s4 * exp(lg);
  }
  const double w = 1.0 - z;
  const double scale = fabs(a) + fabs(b) + fabs(c) + 1.0;
  const bool near_int = fabs(s - rint(s)) < 1e-2;
  if (w < 0.25 && w * scale < 0.5 && !near_int) {
    // A&S 15.3.6: 2F1(a,b;c;z) = G1 2F1(a,b;a+b-c+1;w) + w^s G2 2F1(c-a,c-b;s+1;w)
    double sg[4];
    const double l1 = lgamma_signed(c, &sg[0]) + lgamma_signed(s, &sg[1]) - lgamma_signed(c - a, &sg[2]) -
                      lgamma_signed(c - b, &sg[3]);
    const double g1 = (sg[2] == 0.0 || sg[3] == 0.0) ? 0.0 : sg[0] * sg[1] * sg[2] * sg[3] * exp(l1);
    double tg[4];
    const double l2 = lgamma_signed(c, &tg[0]) + lgamma_signed(-s, &tg[1]) - lgamma_signed(a, &tg[2]) -
                      lgamma_signed(b, &tg[3]);
    const double g2 = (tg[2] == 0.0 || tg[3] == 0.0) ? 0.0 : tg[0] * tg[1] * tg[2] * tg[3] * exp(l2);
    double out = 0.0;
    if (g1 != 0.0) out += g1 * hyp2f1_series(a, b, 1.0 - s, w, ok);
    if (g2 != 0.0) out += g2 * pow(w, s) * hyp2f1_series(c - a, c - b, s + 1.0, w, ok);
    return out;
  }
  return hyp2f1_series(a, b, c, z, ok);
}

__global__ void tau_F_kernel(const double* __restrict__ r, int nr, int Lmin, int Lmax, int nmax_F, int nL,
                             double ns, double pref, double* __restrict__ F, int* __restrict__ err) {
  const int64_t per_n = int64_t(nL) * nr * nr;
  const int64_t total = per_n * (2 * nmax_F + 1);
  const int min_L = Lmin - nmax_F > 0 ? Lmin - nmax_F : 0;
  const int max_L = Lmax + nmax_F + 1;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total; t += int64_t(gridDim.x) * blockDim.x) {
    const int n = int(t / per_n) - nmax_F;
    const int64_t rem = t % per_n;
    const int L = int(rem / (int64_t(nr) * nr));
    const int ir = int((rem / nr) % nr), jr = int(rem % nr);
    if (L < min_L || L >= max_L || L + n < 1 || L < 1 || L + n > Lmax + nmax_F) continue;
    const double i1 = L + (n - 1.0 + ns) / 2.0;
    const double ri = r[ir], rj = r[jr];
    int ok = 1;
    double v;
    if (ri <= rj) {
      const double i2 = (ns - 2.0 - n) / 2.0, i3 = L + 1.5;
      const double pf = pref * exp(lgamma(i1) - lgamma(1.0 - i2) - lgamma(i3));
      v = pf * hyp2f1(i1, i2, i3, ri * ri / (rj * rj), &ok) * pow(ri / rj, double(L)) * pow(rj, 1.0 - ns);
    } else {
      const double i2 = (ns - 2.0 + n) / 2.0, i3 = L + n + 1.5;
      const double pf = pref * exp(lgamma(i1) - lgamma(1.0 - i2) - lgamma(i3));
      v = pf * hyp2f1(i1, i2, i3, rj * rj / (ri * ri), &ok) * pow(rj / ri, double(L + n)) * pow(ri, 1.0 - ns);
    }
    F[t] = v;
    if (!ok) atomicExch(err, 1);
  }
}

template <bool DOT>
__global__ void __launch_bounds__(TAU_THREADS) tau_conv_kernel(
    const double2* __restrict__ X, const double2* __restrict__ A, const int* __restrict__ lm_L,
    const double* __restrict__ lm_w, const double* __restrict__ F, const double* __restrict__ w, int nr, int nL,
    int64_t nlm, double2* __restrict__ out, double* __restrict__ partial) {
  extern __shared__ double2 xs[];  // [nr][TAU_TILE]
  __shared__ double red[TAU_THREADS / 32];
  const int tx = threadIdx.x % TAU_TILE, ty = threadIdx.x / TAU_TILE;
  const int64_t lm = int64_t(blockIdx.x) * TAU_TILE + tx;
  const bool valid = lm < nlm;
  for (int k = ty; k < nr; k += TAU_JLANES)
    xs[k * TAU_TILE + tx] = valid ? __ldg(X + int64_t(k) * nlm + lm) : make_double2(0.0, 0.0);
  __syncthreads();
  const int L = valid ? __ldg(lm_L + lm) : -1;
  const double inv_s4pi = 0.28209479177387814347;  // 1 / sqrt(4 pi)
  double dot = 0.0;
  for (int j = ty; j < nr; j += TAU_JLANES) {
    double sx = 0.0, sy = 0.0;
    if (L >= 0) {
      // F is stored [j][k][L]: the lanes of a warp (consecutive lm, mostly consecutive L) read
      // consecutive words
      const double* Fr = F + int64_t(j) * nr * nL + L;
      for (int k = 0; k < nr; ++k) {
        const double wk = __ldg(w + k);
        if (wk == 0.0) continue;
        const double f = __ldg(Fr + int64_t(k) * nL) * wk;
        const double2 x = xs[k * TAU_TILE + tx];
        sx += f * x.x * inv_s4pi;
        sy += f * x.y * inv_s4pi;
      }
    }
    if (out && valid) out[int64_t(j) * nlm + lm] = make_double2(sx, sy);
    if (DOT && L >= 0) {
      const double wj = __ldg(w + j);
      if (wj != 0.0) {
        const double2 a = __ldg(A + int64_t(j) * nlm + lm);
        dot += __ldg(lm_w + lm) * wj * (a.x * sx + a.y * sy);
      }
    }
  }
  if (DOT) {
    for (int o = 16; o > 0; o >>= 1) dot += __shfl_down_sync(0xffffffffu, dot, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = dot;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int i = 0; i < TAU_THREADS / 32; ++i) s += red[i];
      partial[blockIdx.x] = s;
    }
  }
}

__global__ void tau_partial_sum(const double* __restrict__ partial, int64_t n, double* __restrict__ out) {
  __shared__ double red[256];
  double s = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) s += partial[i];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (int(threadIdx.x) < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = red[0];
}

}  // namespace
}  // namespace ps

using namespace ps;

extern "C" int ps_tau_F_integral(const double* r_arr, int nr, int Lmin, int Lmax, int nmax_F, int nL, double ns,
                                 double pref, double* F, int* err, cudaStream_t stream) {
  if (!r_arr || !F || !err || nr <= 0 || Lmin < 0 || Lmax < Lmin || nmax_F < 0 || nL < Lmax + nmax_F + 1)
    return PS_ERR_INVALID;
  const int64_t total = int64_t(2 * nmax_F + 1) * nL * nr * nr;
  StatScope sc(PS_K_VECTOR, 0.0, 8.0 * double(total), stream);
  int64_t g = (total + 127) / 128;
  if (g > 65535) g = 65535;
  tau_F_kernel<<<int(g), 128, 0, stream>>>(r_arr, nr, Lmin, Lmax, nmax_F, nL, ns, pow(2.0, ns - 3.0) * pref, F,
                                           err);
  PS_LAUNCH_CHECK();
  return PS_OK;
}

extern "C" int ps_tau_convolve_workspace_bytes(int64_t nlm, size_t* bytes) {
  if (!bytes || nlm <= 0) return PS_ERR_INVALID;
  *bytes = sizeof(double) * size_t((nlm + TAU_TILE - 1) / TAU_TILE);
  return PS_OK;
}

extern "C" int ps_tau_convolve_F(const double* X, const double* A, const int* lm_L, const double* lm_w,
                                 const double* F, int nL, const double* r_weights, int nr, int64_t nlm, double* out,
                                 double* dot, void* workspace, size_t workspace_bytes, cudaStream_t stream) {
  if (!X || !lm_L || !F || !r_weights || nr <= 0 || nr > 384 || nL <= 0 || nlm <= 0 || (!out && !dot))
    return PS_ERR_INVALID;
  if (dot && (!A || !lm_w)) return PS_ERR_INVALID;
  const int64_t nblk = (nlm + TAU_TILE - 1) / TAU_TILE;
  if (nblk > 2147483647LL) return PS_ERR_INVALID;
  if (dot && (!workspace || workspace_bytes < sizeof(double) * size_t(nblk))) return PS_ERR_WORKSPACE;
  const size_t smem = sizeof(double2) * size_t(nr) * TAU_TILE;
  StatScope sc(PS_K_VECTOR, 8.0 * double(nlm) * nr * nr, 16.0 * double(nlm) * nr * (out ? 2.0 : 1.0),
               stream);
  if (dot) {
    if (smem > 48 * 1024)
      cudaFuncSetAttribute(tau_conv_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    tau_conv_kernel<true><<<unsigned(nblk), TAU_THREADS, smem, stream>>>(
        reinterpret_cast<const double2*>(X), reinterpret_cast<const double2*>(A), lm_L, lm_w, F, r_weights, nr,
        nL, nlm, reinterpret_cast<double2*>(out), static_cast<double*>(workspace));
    PS_LAUNCH_CHECK();
    tau_partial_sum<<<1, 256, 0, stream>>>(static_cast<double*>(workspace), nblk, dot);
  } else {
    if (smem > 48 * 1024)
      cudaFuncSetAttribute(tau_conv_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    tau_conv_kernel<false><<<unsigned(nblk), TAU_THREADS, smem, stream>>>(
        reinterpret_cast<const double2*>(X), nullptr, lm_L, nullptr, F, r_weights, nr, nL, nlm,
        reinterpret_cast<double2*>(out), nullptr);
  }
  PS_LAUNCH_CHECK();
  return PS_OK;
}
