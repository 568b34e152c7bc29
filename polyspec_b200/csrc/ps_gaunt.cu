// Table evaluation of the small-momentum 3j symbols and Gaunt coefficients of
// ps_gaunt.cuh (used by the parity tests of the direction-dependent contractions).
#include "ps_common.cuh"
#include "ps_gaunt.cuh"
#include "ps_stats.cuh"

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

// ---------------------------------------------------------------------------------
// compute_pF_map_real (polyspec/cython/tauNL_utils.pyx:1531-1620): out[u][i] += Sum over
// shifts Delta (parity of n1) of the Gaunt-weighted inputs at (l + Delta, m -+ mu1) times
// p_{l,l+Delta}^u(r_j) w_j, summed over the radial samples; a gather per (source lm, u).
// Inputs plus/minus are complex [nlm(lmax_in)][nin] with the radial index j reading column
// j of the inputs and sample inds[j] of p.
namespace ps {
namespace {

__global__ void pF_map_kernel(const double2* __restrict__ plus, const double2* __restrict__ minus, int lmax_in,
                              int nin, const double* __restrict__ p, int nshift, int lsize, int npol, int nrp,
                              const double* __restrict__ w, const int* __restrict__ inds, const int* __restrict__ ls,
                              const int* __restrict__ ms, int64_t nl, int n1, int mu1, int nmax,
                              double2* __restrict__ out) {
  const int64_t total = nl * npol;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total; t += int64_t(gridDim.x) * blockDim.x) {
    const int64_t i = t % nl;
    const int u = int(t / nl);
    const int l = ls[i], m = ms[i];
    double2 acc = make_double2(0., 0.);
    for (int Delta = -n1; Delta <= n1; Delta += 2) {
      const int lp = l + Delta;
      if (lp > lmax_in || lp < 0) continue;
      // i^Delta
      const int q = ((Delta % 4) + 4) % 4;
      const double2 iD = q == 0 ? make_double2(1., 0.) : q == 1 ? make_double2(0., 1.)
                       : q == 2 ? make_double2(-1., 0.) : make_double2(0., -1.);
      const double* pp = p + ((int64_t(nmax + Delta) * lsize + l) * npol + u) * nrp;
      for (int part = 0; part < 2; ++part) {
        if (part == 1 && mu1 == 0) break;
        const int mp = part == 0 ? m - mu1 : m + mu1;
        if (abs(mp) > lp) continue;
        const int64_t idx = int64_t(abs(mp)) * (2 * lmax_in + 1 - abs(mp)) / 2 + lp;
        double G, sgn;
        if (part == 0) {
          G = gaunt_small(l, lp, n1, m, -mp, -mu1);
          sgn = (m & 1) ? -0.5 : 0.5;
        } else {
          G = gaunt_small(l, lp, n1, m, -mp, mu1);
          sgn = ((n1 + mu1 + m) & 1) ? -0.5 : 0.5;
        }
        if (G == 0.0) continue;
        double2 gp = make_double2(iD.x * sgn * G, iD.y * sgn * G);
        // part 0: mp >= 0 reads plus, mp < 0 reads conj(minus) times (-1)^mp; part 1 (mp > 0) reads minus
        const bool conj_branch = part == 0 && mp < 0;
        const double2* src = (part == 0 && !conj_branch) ? plus : minus;
        if (conj_branch && (mp & 1)) gp = make_double2(-gp.x, -gp.y);
        double2 s = make_double2(0., 0.);
        for (int j = 0; j < nin; ++j) {
          const double wj = w[j];
          if (wj == 0.0) continue;
          double2 v = src[idx * nin + j];
          if (conj_branch) v.y = -v.y;
          const double f = pp[inds[j]] * wj;
          s.x += v.x * f;
          s.y += v.y * f;
        }
        acc.x += gp.x * s.x - gp.y * s.y;
        acc.y += gp.x * s.y + gp.y * s.x;
      }
    }
    out[int64_t(u) * nl + i].x += acc.x;
    out[int64_t(u) * nl + i].y += acc.y;
  }
}

// out[r][pix] = Sum_i w_i [Re(P[pq_i][0] F[f_i][0]) + 2 Sum_{mu >= 1} Re(P[pq_i][mu] F[f_i][mu])]
// (compute_productPnmu_sym_all, ideal_fisher.pyx:195-212); P [nP][n1+1][npix_tot], F [nF][n1+1][npix_tot]
__global__ void pnmu_sym_kernel(const double2* __restrict__ P, const double2* __restrict__ F, int n1, int64_t ntot,
                                const double* __restrict__ wts, const int* __restrict__ pq, const int* __restrict__ fi,
                                int nw, double* __restrict__ out) {
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < ntot; t += int64_t(gridDim.x) * blockDim.x) {
    double s = 0.0;
    for (int k = 0; k < nw; ++k) {
      const double2* p = P + int64_t(pq[k]) * (n1 + 1) * ntot + t;
      const double2* f = F + int64_t(fi[k]) * (n1 + 1) * ntot + t;
      double2 a = p[0], b = f[0];
      s += wts[k] * (a.x * b.x - a.y * b.y);
      for (int mu = 1; mu <= n1; ++mu) {
        a = p[int64_t(mu) * ntot];
        b = f[int64_t(mu) * ntot];
        s += 2. * wts[k] * (a.x * b.x - a.y * b.y);
      }
    }
    out[t] = s;
  }
}

// out[r][pix] = Sum_i w_i Q[pq_i] F[f_i][mu1] (complex; compute_productQ_complex_all, ideal_fisher.pyx:343-357)
__global__ void q_complex_kernel(const double* __restrict__ Q, const double2* __restrict__ F, int nmu, int mu1,
                                 int64_t ntot, const double* __restrict__ wts, const int* __restrict__ pq,
                                 const int* __restrict__ fi, int nw, double2* __restrict__ out) {
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < ntot; t += int64_t(gridDim.x) * blockDim.x) {
    double2 s = make_double2(0., 0.);
    for (int k = 0; k < nw; ++k) {
      const double q = wts[k] * Q[int64_t(pq[k]) * ntot + t];
      const double2 f = F[(int64_t(fi[k]) * nmu + mu1) * ntot + t];
      s.x += q * f.x;
      s.y += q * f.y;
    }
    out[t] = s;
  }
}

}  // namespace
}  // namespace ps

extern "C" int ps_pF_map_real(const double* plus, const double* minus, int lmax_in, int nin, const double* p,
                              int nshift, int lsize, int npol, int nrp, const double* w, const int* inds,
                              const int* ls, const int* ms, int64_t nl, int n1, int mu1, int nmax, double* out,
                              cudaStream_t stream) {
  if (!plus || !minus || !p || !w || !inds || !ls || !ms || !out || lmax_in < 0 || nin <= 0 || nshift != 2 * nmax + 1 ||
      n1 < 0 || n1 > 16 || n1 > nmax || mu1 < 0 || mu1 > n1 || npol <= 0 || nl <= 0 || nrp <= 0)
    return PS_ERR_INVALID;
  int64_t g = (nl * npol + 127) / 128;
  if (g > 148 * 64) g = 148 * 64;
  pF_map_kernel<<<int(g), 128, 0, stream>>>(reinterpret_cast<const double2*>(plus),
                                            reinterpret_cast<const double2*>(minus), lmax_in, nin, p, nshift, lsize,
                                            npol, nrp, w, inds, ls, ms, nl, n1, mu1, nmax,
                                            reinterpret_cast<double2*>(out));
  PS_LAUNCH_CHECK();
  return PS_OK;
}

extern "C" int ps_product_pnmu_sym(const double* P, const double* F, int n1, int64_t ntot, const double* wts,
                                   const int* pq, const int* fi, int nw, double* out, cudaStream_t stream) {
  if (!P || !F || !wts || !pq || !fi || !out || n1 < 0 || ntot <= 0 || nw <= 0) return PS_ERR_INVALID;
  int64_t g = (ntot + 255) / 256;
  if (g > 148 * 16) g = 148 * 16;
  pnmu_sym_kernel<<<int(g), 256, 0, stream>>>(reinterpret_cast<const double2*>(P), reinterpret_cast<const double2*>(F),
                                              n1, ntot, wts, pq, fi, nw, out);
  PS_LAUNCH_CHECK();
  return PS_OK;
}

extern "C" int ps_product_q_complex(const double* Q, const double* F, int nmu, int mu1, int64_t ntot, const double* wts,
                                    const int* pq, const int* fi, int nw, double* out, cudaStream_t stream) {
  if (!Q || !F || !wts || !pq || !fi || !out || nmu <= 0 || mu1 < 0 || mu1 >= nmu || ntot <= 0 || nw <= 0)
    return PS_ERR_INVALID;
  int64_t g = (ntot + 255) / 256;
  if (g > 148 * 16) g = 148 * 16;
  q_complex_kernel<<<int(g), 256, 0, stream>>>(Q, reinterpret_cast<const double2*>(F), nmu, mu1, ntot, wts, pq, fi, nw,
                                               reinterpret_cast<double2*>(out));
  PS_LAUNCH_CHECK();
  return PS_OK;
}

// ---------------------------------------------------------------------------------
// The n > 0 contractions of the direction-dependent tauNL estimators:
//  * tau_sum_general (polyspec/cython/tauNL_utils.pyx:650-715): Sum over (Delta, mu), (L, M),
//    mu1 and (r_j, r_k) of Re(pref * B[..][(L+Delta, -M-mu)][k] w_k A[n1+mu1][(L, M)][j]) F w_j with
//    pref = (2 if M != 0) i^Delta Gaunt(L, L+Delta, n; M, -M-mu, mu) (n1 n3 n; mu1 mu3 mu) and the
//    conjugate, sign-flipped B where -M-mu < 0; per-CTA partials summed in a fixed order.
//  * convolve_F_general (:1069-1180): for each ((L, M), r_j) the two Gaunt-weighted F convolutions
//    of the shifted [P Q] vectors (M -> M - mu and -M - mu), accumulated as plus + minus and
//    plus - minus at the row of (L, M) in the l <= nLmax list.
// Arrays are [mu][row][r] over a list of (L, M) rows (rowL, rowM); row_of_full maps the m-major
// index of (L, |M|), L <= nLmax, to its row (-1: absent).  F comes transposed, [Delta][L][r'][r], so that
// the lanes of a warp (one radial sample r each) read consecutive addresses.
namespace ps {
namespace {

__device__ __forceinline__ double2 ipow(int d) {
  const int q = ((d % 4) + 4) % 4;
  return q == 0 ? make_double2(1., 0.) : q == 1 ? make_double2(0., 1.) : q == 2 ? make_double2(-1., 0.)
                                                                              : make_double2(0., -1.);
}
__device__ __forceinline__ double2 cm(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ int64_t lm_full(int L, int M, int lmax) {
  return int64_t(M) * (2 * lmax + 1 - M) / 2 + L;
}

// Both kernels give one warp to each (L, M) row.  A row's coupling terms, (Delta, mu, mu1) for the
// tau sum and (Delta, mu, part) for the convolution, are built 32 at a time, one per lane (its
// Gaunt and 3j coefficients, the (L+Delta, -M-mu) or (L+Delta, M-mu) row and which [P Q] plane,
// conjugated or not, it reads) and kept in shared memory; then lane j takes radial sample j and runs
// the r' sum of every term of the batch.  The coefficients are thus computed once per row, not
// once per (row, r), and the terms are visited in (Delta, mu, mu1 / part) order.
constexpr int kRowWarps = 4;
constexpr int kMaxT3 = 33 * 33;  // (2 n1 + 1)(2 n + 1) for n1, n <= 16

// Gaunt coefficients of every (L, M) row: gtab[row][(Delta + n) / 2][mu + n][part] with
// part 0 = Gaunt(L, L+Delta, n; -M, M-mu, mu), part 1 = Gaunt(L, L+Delta, n; M, -M-mu, mu), 0 where
// L+Delta lies outside [Lmin, Lmax] or the M' index outside L+Delta.  They depend on neither mu1,
// the maps nor the weights, so one table serves every contraction of a given n.
__global__ void gaunt_row_table_kernel(const int* __restrict__ rowL, const int* __restrict__ rowM, int nrow, int Lmin,
                                       int Lmax, int n, double* __restrict__ out) {
  const int nmu = 2 * n + 1, per = (n + 1) * nmu * 2;
  const int64_t total = int64_t(nrow) * per;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total; t += int64_t(gridDim.x) * blockDim.x) {
    const int64_t i = t / per;
    const int r = int(t % per), part = r & 1, mu = (r >> 1) % nmu - n, Delta = 2 * ((r >> 1) / nmu) - n;
    const int L = rowL[i], M = rowM[i], Lp = L + Delta;
    const int Mp = part == 0 ? M - mu : -M - mu;
    double G = 0.0;
    if (L >= Lmin && L <= Lmax && Lp >= Lmin && Lp <= Lmax && abs(Mp) <= Lp)
      G = part == 0 ? gaunt_small(L, Lp, n, -M, M - mu, mu) : gaunt_small(L, Lp, n, M, -M - mu, mu);
    out[t] = G;
  }
}

struct RowTerm {
  double2 g;   // complex coefficient
  int rowp;    // source row (-1: the term vanishes)
  int plane;   // source [P Q] / B plane
  int conj;    // read the conjugate of the source
  int dF;      // Delta (F plane nmax_F + Delta)
  int extra;   // tau sum: A plane n1 + mu1; convolution: 0 plus part, 1 minus part
};

// Source vectors of up to kStage terms, radial samples k0 .. k0 + kn - 1, staged in shared memory
// (conjugated where the term says so) by coalesced loads that are all in flight together; the r'
// sums then read them as broadcasts.
constexpr int kStage = 8;

__device__ __forceinline__ void stage_sources(const double2* __restrict__ src, const RowTerm* terms, int qn, int nrow,
                                              int nr, int k0, int kn, int lane, double2 (*vs)[32]) {
#pragma unroll
  for (int qq = 0; qq < kStage; ++qq) {
    if (qq < qn && terms[qq].rowp >= 0 && lane < kn) {
      double2 v = src[(int64_t(terms[qq].plane) * nrow + terms[qq].rowp) * nr + k0 + lane];
      if (terms[qq].conj) v.y = -v.y;
      vs[qq][lane] = v;
    }
  }
}

// s += Sum_k v[k] F_j(r'_k) w_k over kn samples (F read at inds[k] when given), skipping zero weights
// as the reference does, in the order of k; Fp, ld, jc as for radial_sum_list.
__device__ __forceinline__ void radial_sum(const double2* v, const double* __restrict__ Fp, int64_t ld, int jc,
                                           const int* __restrict__ inds, const double* __restrict__ w, int kn,
                                           double2& s) {
  for (int k = 0; k < kn; ++k) {
    const double wk = w[k];
    if (wk == 0.0) continue;
    const double2 x = v[k];
    const double f = Fp[(inds ? inds[k] : k) * ld + jc] * wk;
    s.x += x.x * f;
    s.y += x.y * f;
  }
}

// The radial samples with non-zero weight, in order, for N_r <= 32 (one staging chunk): their
// index k, weight and F column (inds[k], or k); built once per block.
struct RadialList {
  int nk;
  int k[32];
  int col[32];
  double w[32];
};

__device__ __forceinline__ void build_radial_list(RadialList& rl, const double* __restrict__ w,
                                                  const int* __restrict__ inds, int nr) {
  if (threadIdx.x == 0) {
    int c = 0;
    for (int k = 0; k < nr && k < 32; ++k) {
      if (w[k] == 0.0) continue;
      rl.k[c] = k;
      rl.col[c] = inds ? inds[k] : k;
      rl.w[c] = w[k];
      ++c;
    }
    rl.nk = c;
  }
}

// s += Sum over the listed samples of v[k] F_j(col) w, the same terms in the same order as radial_sum.
// Fp is the (Delta, L) plane of the transposed F, [r'][r] with row stride ld, jc the lane's column.
__device__ __forceinline__ void radial_sum_list(const double2* v, const double* __restrict__ Fp, int64_t ld, int jc,
                                                const RadialList& rl, double2& s) {
  const int nk = rl.nk;
  for (int q = 0; q < nk; ++q) {
    const double2 x = v[rl.k[q]];
    const double f = Fp[rl.col[q] * ld + jc] * rl.w[q];
    s.x += x.x * f;
    s.y += x.y * f;
  }
}

// The coupling term t of row (L, M), built out of line so that its Gaunt and 3j evaluation does not
// raise the register count of the r' loops.
__device__ __noinline__ RowTerm tau_term(int t, int nT, int L, int M, const int* __restrict__ row_of_full, int nLmax,
                                         int Lmin, int Lmax, int n1, int n3, int n, const double* __restrict__ grow,
                                         const double* t3tab) {
  RowTerm c;
  c.rowp = -1;
  if (t >= nT) return c;
  const int nmu = 2 * n + 1, nmu1 = 2 * n1 + 1;
  const int mu1 = t % nmu1 - n1;
  const int mu = (t / nmu1) % nmu - n;
  const int Delta = 2 * (t / (nmu1 * nmu)) - n;
  const int Lp = L + Delta, Mp = -M - mu, mu3 = -mu1 - mu;
  if (Lp < Lmin || Lp > Lmax || abs(Mp) > Lp || abs(mu3) > n3) return c;
  const double G = grow[(((Delta + n) / 2) * nmu + mu + n) * 2 + 1];
  double t3 = G != 0.0 ? t3tab[(mu1 + n1) * nmu + mu + n] : 0.0;
  const int rowp = row_of_full[lm_full(Lp, abs(Mp), nLmax)];
  if (t3 == 0.0 || rowp < 0) return c;
  if (Mp < 0 && ((Mp + n3 + mu3) & 1)) t3 = -t3;
  const double2 p1 = cm(ipow(Delta), make_double2((M != 0 ? 2.0 : 1.0) * G, 0.));
  c.g = make_double2(p1.x * t3, p1.y * t3);
  c.rowp = rowp;
  c.plane = Mp >= 0 ? n3 + mu3 : n3 - mu3;
  c.conj = Mp < 0;
  c.dF = Delta;
  c.extra = n1 + mu1;
  return c;
}

__device__ __noinline__ RowTerm conv_term(int t, int nT, int L, int M, const int* __restrict__ row_of_full, int nLmax,
                                          int Lmin, int Lmax, int n1, int n3, int n, int mu1,
                                          const double* __restrict__ grow, const double* t3tab) {
  RowTerm c;
  c.rowp = -1;
  if (t >= nT) return c;
  const int nmu = 2 * n + 1;
  const int part = t & 1;
  const int mu = (t >> 1) % nmu - n;
  const int Delta = 2 * ((t >> 1) / nmu) - n;
  const int Lp = L + Delta, mu3 = -mu1 - mu;
  const int Mp = part == 0 ? M - mu : -M - mu;
  if (Lp < Lmin || Lp > Lmax || abs(mu3) > n3 || (part == 1 && M == 0) || abs(Mp) > Lp) return c;
  const double t3 = t3tab[(mu1 + n1) * nmu + mu + n];
  double G = t3 != 0.0 ? grow[(((Delta + n) / 2) * nmu + mu + n) * 2 + part] : 0.0;
  const int rowp = row_of_full[lm_full(Lp, abs(Mp), nLmax)];
  if (G == 0.0 || rowp < 0) return c;
  const double2 pref = make_double2(ipow(Delta).x * t3, ipow(Delta).y * t3);
  if (part == 0) {
    const int e = Mp >= 0 ? M : (M + Mp + n3 + mu3);
    if (e & 1) G = -G;
    if (M != 0) G *= 0.5;
    c.g = make_double2(pref.x * G, pref.y * G);
  } else {
    if (Mp < 0 && ((Mp + n3 + mu3) & 1)) G = -G;
    G *= 0.5;
    c.g = make_double2(pref.x * G, -pref.y * G);  // conj(pref)
  }
  c.rowp = rowp;
  c.plane = Mp >= 0 ? n3 + mu3 : n3 - mu3;
  // plus part reads PQ[n3+mu3] (Mp >= 0) or conj(PQ[n3-mu3]); minus part the conjugates of those
  c.conj = (part == 0) ? (Mp < 0) : (Mp >= 0);
  c.dF = Delta;
  c.extra = part;
  return c;
}

__global__ void __launch_bounds__(32 * kRowWarps)
tau_general_kernel(const double2* __restrict__ A, const double2* __restrict__ B, const int* __restrict__ row_of_full,
                   const int* __restrict__ rowL, const int* __restrict__ rowM, int nrow, int nLmax, int Lmin,
                   int Lmax, const double* __restrict__ F, int nLF, int nmax_F, const double* __restrict__ w, int nr,
                   int n1, int n3, int n, const double* __restrict__ gtab, double* __restrict__ partial) {
  __shared__ RowTerm sh[kRowWarps][32];
  __shared__ double2 vsh[kRowWarps][kStage][32];
  __shared__ double red[32 * kRowWarps];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  RowTerm* terms = sh[wid];
  const int nmu = 2 * n + 1, nmu1 = 2 * n1 + 1;
  const int nT = (n + 1) * nmu * nmu1;  // Delta = -n, -n + 2, ..., n (odd Delta + n: no Gaunt coupling)
  __shared__ double t3tab[kMaxT3];
  __shared__ RadialList rl;
  for (int q = threadIdx.x; q < nmu1 * nmu; q += blockDim.x)
    t3tab[q] = threej_small(n1, n3, n, q / nmu - n1, -(q / nmu - n1) - (q % nmu - n), q % nmu - n);
  build_radial_list(rl, w, nullptr, nr);
  __syncthreads();
  double acc = 0.0;
  for (int64_t i = blockIdx.x * int64_t(kRowWarps) + wid; i < nrow; i += int64_t(gridDim.x) * kRowWarps) {
    const int L = rowL[i], M = rowM[i];
    if (L < Lmin || L > Lmax) continue;  // warp-uniform
    for (int j0 = 0; j0 < nr; j0 += 32) {
      const int j = j0 + lane;
      const double wj = j < nr ? w[j] : 0.0;
      for (int t0 = 0; t0 < nT; t0 += 32) {
        const RowTerm c = tau_term(t0 + lane, nT, L, M, row_of_full, nLmax, Lmin, Lmax, n1, n3, n,
                                   gtab + i * int64_t((n + 1) * nmu * 2), t3tab);
        terms[lane] = c;
        __syncwarp();
        const int nt = min(32, nT - t0);
        for (int q0 = 0; q0 < nt; q0 += kStage) {
          const int qn = min(kStage, nt - q0);
          double2 sacc[kStage];
#pragma unroll
          for (int qq = 0; qq < kStage; ++qq) sacc[qq] = make_double2(0., 0.);
          for (int k0 = 0; k0 < nr; k0 += 32) {
            const int kn = min(32, nr - k0);
            stage_sources(B, terms + q0, qn, nrow, nr, k0, kn, lane, vsh[wid]);
            __syncwarp();
            if (wj != 0.0) {
#pragma unroll
              for (int qq = 0; qq < kStage; ++qq) {
                if (qq < qn && terms[q0 + qq].rowp >= 0) {
                  const double* Fp = F + (int64_t(nmax_F + terms[q0 + qq].dF) * nLF + L) * nr * nr;
                  if (nr <= 32)
                    radial_sum_list(vsh[wid][qq], Fp, nr, j, rl, sacc[qq]);
                  else
                    radial_sum(vsh[wid][qq], Fp + int64_t(k0) * nr, nr, j, nullptr, w + k0, kn, sacc[qq]);
                }
              }
            }
            __syncwarp();
          }
          if (wj != 0.0) {
#pragma unroll
            for (int qq = 0; qq < kStage; ++qq) {
              if (qq < qn && terms[q0 + qq].rowp >= 0) {
                const RowTerm& tm = terms[q0 + qq];
                const double2 v = cm(tm.g, sacc[qq]);
                const double2 a = A[(int64_t(tm.extra) * nrow + i) * nr + j];
                acc += (v.x * a.x - v.y * a.y) * wj;
              }
            }
          }
        }
        __syncwarp();
      }
    }
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (int(threadIdx.x) < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

__global__ void sum_partials(const double* __restrict__ partial, int64_t n, double* __restrict__ out) {
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

__global__ void __launch_bounds__(32 * kRowWarps)
conv_general_kernel(const double2* __restrict__ PQ, const int* __restrict__ row_of_full, const int* __restrict__ rowL,
                    const int* __restrict__ rowM, const int* __restrict__ full_of_row, int nrow, int nLmax, int Lmin,
                    int Lmax, const double* __restrict__ F, int nLF, int nrF, int nmax_F, const double* __restrict__ w,
                    const int* __restrict__ inds, int nr, int n1, int n3, int n, int mu1,
                    const double* __restrict__ gtab, double2* __restrict__ out_re, double2* __restrict__ out_im) {
  __shared__ RowTerm sh[kRowWarps][32];
  __shared__ double2 vsh[kRowWarps][kStage][32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  RowTerm* terms = sh[wid];
  const int nmu = 2 * n + 1;
  const int nT = (n + 1) * nmu * 2;  // (Delta, mu, part), part 0: M -> M - mu, part 1: M -> -M - mu
  __shared__ double t3tab[kMaxT3];
  __shared__ RadialList rl;
  for (int q = threadIdx.x; q < (2 * n1 + 1) * nmu; q += blockDim.x)
    t3tab[q] = threej_small(n1, n3, n, q / nmu - n1, -(q / nmu - n1) - (q % nmu - n), q % nmu - n);
  build_radial_list(rl, w, inds, nr);
  __syncthreads();
  for (int64_t i = blockIdx.x * int64_t(kRowWarps) + wid; i < nrow; i += int64_t(gridDim.x) * kRowWarps) {
    const int L = rowL[i], M = rowM[i], fo = full_of_row[i];
    if (L < Lmin || L > Lmax || fo < 0) continue;  // warp-uniform
    for (int j0 = 0; j0 < nr; j0 += 32) {
      const int j = j0 + lane;
      const bool active = j < nr;
      const int ij = active ? inds[j] : 0;
      double2 plus = make_double2(0., 0.), minus = plus;
      for (int t0 = 0; t0 < nT; t0 += 32) {
        const RowTerm c = conv_term(t0 + lane, nT, L, M, row_of_full, nLmax, Lmin, Lmax, n1, n3, n, mu1,
                                    gtab + i * int64_t(nT), t3tab);
        terms[lane] = c;
        __syncwarp();
        const int nt = min(32, nT - t0);
        for (int q0 = 0; q0 < nt; q0 += kStage) {
          const int qn = min(kStage, nt - q0);
          double2 sacc[kStage];
#pragma unroll
          for (int qq = 0; qq < kStage; ++qq) sacc[qq] = make_double2(0., 0.);
          for (int k0 = 0; k0 < nr; k0 += 32) {
            const int kn = min(32, nr - k0);
            stage_sources(PQ, terms + q0, qn, nrow, nr, k0, kn, lane, vsh[wid]);
            __syncwarp();
            if (active) {
#pragma unroll
              for (int qq = 0; qq < kStage; ++qq) {
                if (qq < qn && terms[q0 + qq].rowp >= 0) {
                  const double* Fp = F + (int64_t(nmax_F + terms[q0 + qq].dF) * nLF + L) * nrF * nrF;
                  if (nr <= 32)
                    radial_sum_list(vsh[wid][qq], Fp, nrF, ij, rl, sacc[qq]);
                  else
                    radial_sum(vsh[wid][qq], Fp, nrF, ij, inds + k0, w + k0, kn, sacc[qq]);
                }
              }
            }
            __syncwarp();
          }
          if (active) {
#pragma unroll
            for (int qq = 0; qq < kStage; ++qq) {
              if (qq < qn && terms[q0 + qq].rowp >= 0) {
                const double2 r = cm(sacc[qq], terms[q0 + qq].g);
                if (terms[q0 + qq].extra == 0) {
                  plus.x += r.x;
                  plus.y += r.y;
                } else {
                  minus.x += r.x;
                  minus.y += r.y;
                }
              }
            }
          }
        }
        __syncwarp();
      }
      if (active) {
        const int64_t o = int64_t(fo) * nr + j;
        out_re[o].x += plus.x + minus.x;
        out_re[o].y += plus.y + minus.y;
        out_im[o].x += plus.x - minus.x;
        out_im[o].y += plus.y - minus.y;
      }
    }
  }
}

}  // namespace
}  // namespace ps

// CTAs of the per-row contraction kernels: one per kRowWarps rows, at most 16 per SM of
// the current device.  ps_tau_general_workspace_bytes and the launches both size by this
// one function (one partial sum per CTA).
static int64_t row_grid(int nrow) {
  const int64_t cap = int64_t(ps::device_sms()) * 16;
  int64_t g = (int64_t(nrow) + kRowWarps - 1) / kRowWarps;
  return g > cap ? cap : g;
}

extern "C" int ps_tau_general_workspace_bytes(int nrow, int nr, size_t* bytes) {
  if (!bytes || nrow <= 0 || nr <= 0) return PS_ERR_INVALID;
  *bytes = sizeof(double) * size_t(row_grid(nrow));
  return PS_OK;
}

extern "C" int ps_gaunt_row_table(const int* rowL, const int* rowM, int nrow, int Lmin, int Lmax, int n, double* out,
                                  cudaStream_t stream) {
  if (!rowL || !rowM || !out || nrow <= 0 || n < 0 || n > 16) return PS_ERR_INVALID;
  const int64_t total = int64_t(nrow) * (n + 1) * (2 * n + 1) * 2;
  int64_t g = (total + 255) / 256;
  if (g > 148 * 32) g = 148 * 32;
  gaunt_row_table_kernel<<<int(g), 256, 0, stream>>>(rowL, rowM, nrow, Lmin, Lmax, n, out);
  PS_LAUNCH_CHECK();
  return PS_OK;
}

extern "C" int ps_tau_sum_general(const double* A, const double* B, const int* row_of_full, const int* rowL,
                                  const int* rowM, int nrow, int nLmax, int Lmin, int Lmax, const double* F, int nLF,
                                  int nmax_F, const double* w, int nr, int n1, int n3, int n, const double* gtab,
                                  double* out, void* workspace, size_t workspace_bytes, cudaStream_t stream) {
  if (!A || !B || !row_of_full || !rowL || !rowM || !F || !w || !gtab || !out || nrow <= 0 || nr <= 0 || n < 0 ||
      n > 16 ||
      n1 < 0 || n1 > 16 || n3 < 0 || n3 > 16 || n > nmax_F || Lmax >= nLF || Lmax > nLmax)
    return PS_ERR_INVALID;
  const int64_t nblk = row_grid(nrow);
  if (!workspace || workspace_bytes < sizeof(double) * size_t(nblk)) return PS_ERR_WORKSPACE;
  StatScope sc(PS_K_PIXEL, 0.0, 16.0 * double(nrow) * nr * (2 * n1 + 2 * n3 + 2), stream);
  tau_general_kernel<<<unsigned(nblk), 32 * kRowWarps, 0, stream>>>(
      reinterpret_cast<const double2*>(A), reinterpret_cast<const double2*>(B), row_of_full, rowL, rowM, nrow, nLmax,
      Lmin, Lmax, F, nLF, nmax_F, w, nr, n1, n3, n, gtab, static_cast<double*>(workspace));
  PS_LAUNCH_CHECK();
  sum_partials<<<1, 256, 0, stream>>>(static_cast<double*>(workspace), nblk, out);
  PS_LAUNCH_CHECK();
  return PS_OK;
}

extern "C" int ps_convolve_F_general(const double* PQ, const int* row_of_full, const int* rowL, const int* rowM,
                                     const int* full_of_row, int nrow, int nLmax, int Lmin, int Lmax, const double* F,
                                     int nLF, int nrF, int nmax_F, const double* w, const int* inds, int nr, int n1,
                                     int n3, int n, int mu1, const double* gtab, double* out_re, double* out_im,
                                     cudaStream_t stream) {
  if (!PQ || !row_of_full || !rowL || !rowM || !full_of_row || !F || !w || !inds || !gtab || !out_re || !out_im ||
      nrow <= 0 ||
      nr <= 0 || nrF < nr || n < 0 || n > 16 || n1 < 0 || n1 > 16 || n3 < 0 || n3 > 16 || abs(mu1) > n1 ||
      n > nmax_F || Lmax >= nLF || Lmax > nLmax)
    return PS_ERR_INVALID;
  StatScope sc(PS_K_PIXEL, 0.0, 16.0 * double(nrow) * nr * (2 * n3 + 3), stream);
  conv_general_kernel<<<int(row_grid(nrow)), 32 * kRowWarps, 0, stream>>>(reinterpret_cast<const double2*>(PQ), row_of_full, rowL, rowM,
                                                  full_of_row, nrow, nLmax, Lmin, Lmax, F, nLF, nrF, nmax_F, w, inds,
                                                  nr, n1, n3, n, mu1, gtab, reinterpret_cast<double2*>(out_re),
                                                  reinterpret_cast<double2*>(out_im));
  PS_LAUNCH_CHECK();
  return PS_OK;
}
