// Table evaluation of the small-momentum 3j symbols and Gaunt coefficients of
// ps_gaunt.cuh (used by the parity tests of the direction-dependent contractions).
#include "ps_common.cuh"
#include "ps_gaunt.cuh"

namespace ps {
namespace {

__global__ void gaunt_table_kernel(const int* __restrict__ args, int n, int gaunt, double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int* a = args + 6 * int64_t(i);
  out[i] = gaunt ? gaunt_small(a[0], a[1], a[2], a[3], a[4], a[5]) : threej_small(a[0], a[1], a[2], a[3], a[4], a[5]);
}

}  // namespace
}  // namespace ps

using namespace ps;

extern "C" int ps_gaunt_table(const int* args, int n, int gaunt, double* out, cudaStream_t stream) {
  if (!args || !out || n < 0) return PS_ERR_INVALID;
  if (n == 0) return PS_OK;
  gaunt_table_kernel<<<(n + 127) / 128, 128, 0, stream>>>(args, n, gaunt ? 1 : 0, out);
  PS_LAUNCH_CHECK();
  return PS_OK;
}

// ---------------------------------------------------------------------------------
// shift_and_weight_map_all (polyspec/cython/tauNL_utils.pyx:407-512) as a gather.
//
// For each shift Delta in [-n, n] with Delta + n even, every source (l, m >= 0) of the
// filtered harmonic list feeds up to two targets (L = l + Delta, |mu - m|) and
// (L, mu + m) of the l <= lmax + n list, with the Gaunt coefficient and the reference's
// phase (weight i^Delta (-1)^mu, halved for M != 0, (-1)^(M+Delta) or (-1)^m for the
// conjugate-side terms).  Seen from a target (L, K >= 0) the sources are
//   (a) m = mu - K       (M = K >= 0):       real += in g, imag += in g
//   (b) m = mu + K, K>0  (M = -K < 0):       real += conj(in) g, imag -= conj(in) g
//   (c) m = K - mu > 0   (second term):      real += conj(in) g2, imag += conj(in) g2
// with in[r] = Sum_X flX[nmax + Delta][l][X][r] conj(h[X][src]).  Kernel 1 tabulates the
// (source, coefficient) of (a), (b), (c) per (Delta, target); kernel 2 runs one thread per
// (target, radial sample) and adds the contributions of all shifts.
namespace ps {
namespace {

struct SwTerm {
  int src;     // index into the source lm list, -1: none
  double2 g;   // complex coefficient
};

__device__ __forceinline__ double2 cmulr(double2 a, double r) { return make_double2(a.x * r, a.y * r); }

__global__ void sw_table_kernel(const int* __restrict__ src_of_lm, int lmax_src, const int* __restrict__ tL,
                                const int* __restrict__ tK, int64_t ntarget, int n, int mu, double2 weight,
                                SwTerm* __restrict__ tab) {
  const int nD = n + 1;  // shifts -n, -n+2, ..., n
  const int64_t total = ntarget * nD;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total; t += int64_t(gridDim.x) * blockDim.x) {
    const int64_t it = t % ntarget;
    const int Delta = -n + 2 * int(t / ntarget);
    const int L = tL[it], K = tK[it];
    const int l = L - Delta;
    // pref = weight i^Delta (-1)^mu
    double2 pref = weight;
    const int q = ((Delta % 4) + 4) % 4;
    for (int j = 0; j < q; ++j) pref = make_double2(-pref.y, pref.x);
    if (mu & 1) pref = make_double2(-pref.x, -pref.y);
    SwTerm a{-1, make_double2(0., 0.)}, b = a, c = a;
    const bool lok = l >= 0 && l <= lmax_src;
    auto src_index = [&](int ll, int mm) -> int {
      if (ll < 0 || ll > lmax_src || mm < 0 || mm > ll) return -1;
      return src_of_lm[int64_t(mm) * (2 * lmax_src + 1 - mm) / 2 + ll];
    };
    if (lok) {
      // (a) source m = mu - K >= 0, M = K >= 0 (halved unless M = 0)
      {
        const int m = mu - K, s = src_index(l, m);
        if (s >= 0) {
          const double G = gaunt_small(l, L, n, m, K, -mu);
          a.src = s;
          a.g = cmulr(pref, (K == 0 ? 1.0 : 0.5) * G);
        }
      }
      // (b) source m = mu + K with K > 0, M = -K < 0: factor (-1)^(M + Delta) / 2
      if (K > 0) {
        const int m = mu + K, s = src_index(l, m);
        if (s >= 0) {
          const double G = gaunt_small(l, L, n, m, -K, -mu);
          b.src = s;
          b.g = cmulr(pref, (((-K + Delta) & 1) ? -0.5 : 0.5) * G);
        }
      }
      // (c) source m = K - mu > 0 (the m < 0 half of the source), M = K
      {
        const int m = K - mu, s = src_index(l, m);
        if (m > 0 && s >= 0) {
          double G;
          double2 g;
          if (mu == 0) {  // the reference takes (-1)^Delta times the m >= 0 coefficient of this source
            const double G1 = gaunt_small(l, L, n, m, -m, 0);
            g = cmulr(pref, (((-m + Delta) & 1) ? -0.5 : 0.5) * G1);
            if (Delta & 1) g = make_double2(-g.x, -g.y);
          } else {
            G = gaunt_small(l, L, n, -m, K, -mu);
            g = cmulr(pref, ((m & 1) ? -0.5 : 0.5) * G);
          }
          c.src = s;
          c.g = g;
        }
      }
    }
    tab[3 * t] = a;
    tab[3 * t + 1] = b;
    tab[3 * t + 2] = c;
  }
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__global__ void sw_gather_kernel(const double* __restrict__ flX, int lsize, int npol, int nr, int nmax,
                                 const double2* __restrict__ h, int64_t nsrc, const int* __restrict__ src_l,
                                 const SwTerm* __restrict__ tab, int64_t ntarget, int n, double2* __restrict__ Lre,
                                 double2* __restrict__ Lim) {
  const int64_t total = ntarget * nr;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total; t += int64_t(gridDim.x) * blockDim.x) {
    const int64_t it = t % ntarget;
    const int r = int(t / ntarget);
    double2 re = make_double2(0., 0.), im = re;
    for (int d = 0; d <= n; ++d) {
      const int Delta = -n + 2 * d;
      const SwTerm* T = tab + 3 * (int64_t(d) * ntarget + it);
      for (int w = 0; w < 3; ++w) {
        const int s = T[w].src;
        if (s < 0) continue;
        const int l = src_l[s];
        double2 in = make_double2(0., 0.);
        for (int X = 0; X < npol; ++X) {
          const double f = flX[((int64_t(nmax + Delta) * lsize + l) * npol + X) * nr + r];
          const double2 hv = h[int64_t(X) * nsrc + s];
          in.x += f * hv.x;  // f conj(h)
          in.y -= f * hv.y;
        }
        const double2 g = T[w].g;
        if (w == 0) {  // in g to both
          const double2 v = cmul(in, g);
          re.x += v.x; re.y += v.y; im.x += v.x; im.y += v.y;
        } else if (w == 1) {  // conj(in) g: + real, - imag
          const double2 v = cmul(make_double2(in.x, -in.y), g);
          re.x += v.x; re.y += v.y; im.x -= v.x; im.y -= v.y;
        } else {  // conj(in) g2 to both
          const double2 v = cmul(make_double2(in.x, -in.y), g);
          re.x += v.x; re.y += v.y; im.x += v.x; im.y += v.y;
        }
      }
    }
    const int64_t o = int64_t(r) * ntarget + it;
    Lre[o].x += re.x; Lre[o].y += re.y;
    Lim[o].x += im.x; Lim[o].y += im.y;
  }
}

}  // namespace
}  // namespace ps

extern "C" int ps_shift_weight_workspace_bytes(int64_t ntarget, int n, size_t* bytes) {
  if (!bytes || ntarget <= 0 || n < 0) return PS_ERR_INVALID;
  *bytes = sizeof(SwTerm) * 3 * size_t(ntarget) * size_t(n + 1);
  return PS_OK;
}

extern "C" int ps_shift_weight_map_all(const double* flX, int nshift, int lsize, int npol, int nr, const double* h,
                                       int64_t nsrc, const int* src_l, const int* src_of_lm, int lmax_src,
                                       const int* tL, const int* tK, int64_t ntarget, int n, int mu, double weight_re,
                                       double weight_im, int nmax, double* Lre, double* Lim, void* workspace,
                                       size_t workspace_bytes, cudaStream_t stream) {
  if (!flX || !h || !src_l || !src_of_lm || !tL || !tK || !Lre || !Lim || n < 0 || n > 16 || mu < 0 || mu > n ||
      nmax < n || nshift != 2 * nmax + 1 || npol <= 0 || nr <= 0 || nsrc <= 0 || ntarget <= 0 || lmax_src < 0 ||
      lsize <= lmax_src)
    return PS_ERR_INVALID;
  if (!workspace || workspace_bytes < sizeof(SwTerm) * 3 * size_t(ntarget) * size_t(n + 1)) return PS_ERR_WORKSPACE;
  SwTerm* tab = static_cast<SwTerm*>(workspace);
  int64_t g = (ntarget * (n + 1) + 127) / 128;
  if (g > 148 * 64) g = 148 * 64;
  sw_table_kernel<<<int(g), 128, 0, stream>>>(src_of_lm, lmax_src, tL, tK, ntarget, n, mu,
                                              make_double2(weight_re, weight_im), tab);
  PS_LAUNCH_CHECK();
  g = (ntarget * nr + 127) / 128;
  if (g > 148 * 64) g = 148 * 64;
  sw_gather_kernel<<<int(g), 128, 0, stream>>>(flX, lsize, npol, nr, nmax, reinterpret_cast<const double2*>(h), nsrc,
                                               src_l, tab, ntarget, n, reinterpret_cast<double2*>(Lre),
                                               reinterpret_cast<double2*>(Lim));
  PS_LAUNCH_CHECK();
  return PS_OK;
}
