// Collider tauNL templates (tauNL-light:s,nu_s and tauNL-heavy:s,mu_s of
// polyspec/tspec_template.py), FP64 / complex FP64.
//
//  * ps_kint_collider_jlK: jlK[l][k][r] = j_l(K_k r_r) linearly interpolated from a
//    j_l(x) table (rows tab_lmin..), the interval found as in ps_kint_radial (largest
//    grid point below K r, numpy's searchsorted(...) - 1 in interpolate_jlkr,
//    polyspec/cython/k_integrals.pyx:84-110).  One thread per (k, r) (r fastest), so
//    the writes of each l row are coalesced.
//  * ps_kint_collider_F: F^{betaF}_{L,L+n}(r_i, r_j) = Sum_k (K_k - K_{k-1})(f_{k-1} + f_k),
//    f_k = Kprod_k j_L(K_k r_i) j_{L+n}(K_k r_j) (compute_collider_F_integral,
//    k_integrals.pyx:496-545; Kprod complex, zero beyond K_coll).  One thread per
//    (n, L, i, j) with j fastest: the j_{L+n} reads of a warp are consecutive in the
//    [l][k][r] table and the j_L read is a broadcast.  K is summed in order; n = 0 is
//    computed for j <= i and mirrored, as the reference.
//  * ps_tau_sum_collider_diag: the s = 0 and nu_s = 0 forms (tau_sum_n0_collider and
//    tau_sum_nu0_collider, polyspec/cython/tauNL_utils.pyx:877-964):
//    Sum over rows (L, M), Lmin <= L <= Lmax, of w_M Re(pref Sum_lam Sum_{j,k}
//    F_L(r_j, r_k) w_j w_k A[lam](r_j) conj(B[lam](r_k))), w_M = 1 (M = 0) or 2.
//  * ps_tau_sum_collider_general: tau_sum_general_collider (tauNL_utils.pyx:723-875): the
//    Gaunt- and 3j-weighted sum over S (even, <= 2s), Delta, Lam, lam1 of
//    Re(C_S i^Delta G(L, L+Delta, S; M, M', Lam) (s s S; lam1 lam3 Lam) B_k w_k A_j w_j
//    F_{L,L+Delta}(r_j, r_k)), with the conjugation signs of M' < 0 and, for complex beta,
//    the m -> -m piece.
//    One warp per row: lanes own r_k; for each (Delta, lam1, piece) the lanes first form
//    v_k = Sum_j A_j w_j F_{L,L+Delta}(r_j, r_k) (F rows read coalesced, A broadcast), then
//    every (S, Lam) term adds Re(pref B_k w_k v_k).  Per-block partial sums, then one
//    ordered reduction.
//  * ps_convolve_F_collider: convolve_F_general_collider (tauNL_utils.pyx:1197-1355) for one
//    lam1: the S = 0 term (diagonal in (L, M)) and the S > 0 Gaunt- and 3j-coupled terms of
//    F^beta_{L,L+Delta}(r_j, r_k) [P^beta Q]_{L',M'}(r_k), accumulated as the "plus" (M' = M - Lam)
//    and "minus" (M' = -M - Lam, conjugated F) parts and written as plus + minus, plus - minus
//    into the full l-list.  One warp per row, lanes own the output radial index j.
//  * ps_pF_map_complex: compute_pF_map_complex (tauNL_utils.pyx:1357-1446): the Gaunt-weighted
//    shifts (l + Delta, m - mu1) and (l + Delta, -m - mu1) of the [Q F_PQ] harmonics times the
//    complex p^beta_{l,l+Delta}(r_j) w_j, summed over j.  One thread per (u, l m).
#include "ps_common.cuh"
#include "ps_gaunt.cuh"
#include "ps_stats.cuh"

namespace ps {
namespace {

constexpr int kCollWarps = 8;

__global__ void coll_jlK_kernel(const double* __restrict__ table, const double* __restrict__ xs, int64_t nx, int nl,
                                const double* __restrict__ K, int nK, const double* __restrict__ r, int nr,
                                double* __restrict__ jlK) {
  const int64_t total = int64_t(nK) * nr;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total; t += int64_t(gridDim.x) * blockDim.x) {
    const int ir = int(t % nr);
    const int ik = int(t / nr);
    const double kr = K[ik] * r[ir];
    int64_t lo = 0, hi = nx - 1;
    while (hi - lo > 1) {
      const int64_t mid = (lo + hi) >> 1;
      if (xs[mid] < kr) lo = mid;
      else hi = mid;
    }
    const double dx = xs[lo + 1] - xs[lo];
    const double xp = (xs[lo + 1] - kr) / dx, xm = (kr - xs[lo]) / dx;
    for (int l = 0; l < nl; ++l) {
      const double* row = table + int64_t(l) * nx;
      jlK[(int64_t(l) * nK + ik) * nr + ir] = row[lo] * xp + row[lo + 1] * xm;
    }
  }
}

__global__ void coll_F_kernel(const double* __restrict__ jlK, int nl_tab, int glmin, const double* __restrict__ K,
                              int nK, const double2* __restrict__ Kprod, int nr, int Lmin, int Lmax, int nF, int nLout,
                              double2* __restrict__ out) {
  const int L0 = max(Lmin - nF, 0), L1 = Lmax + nF;
  const int nL = L1 - L0 + 1;
  const int64_t total = int64_t(2 * nF + 1) * nL * nr * nr;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total; t += int64_t(gridDim.x) * blockDim.x) {
    int jr = int(t % nr);
    int ir = int((t / nr) % nr);
    const int L = L0 + int((t / (int64_t(nr) * nr)) % nL);
    const int n = int(t / (int64_t(nr) * nr * nL)) - nF;
    if (L + n < 1 || L < 1 || L + n > Lmax + nF || L >= nLout) continue;
    const int ind1 = L - glmin, ind2 = L - glmin + n;
    if (ind1 < 0 || ind2 < 0 || ind1 >= nl_tab || ind2 >= nl_tab) continue;
    const int64_t o = ((int64_t(nF + n) * nLout + L) * nr + ir) * nr + jr;
    if (n == 0 && jr > ir) {  // mirrored from (jr, ir), as the reference fills it
      const int tmp = ir;
      ir = jr;
      jr = tmp;
    }
    const double* a = jlK + int64_t(ind1) * nK * nr + ir;
    const double* b = jlK + int64_t(ind2) * nK * nr + jr;
    double2 flow = make_double2(Kprod[0].x * a[0] * b[0], Kprod[0].y * a[0] * b[0]);
    double2 acc = make_double2(0.0, 0.0);
    for (int ik = 1; ik < nK; ++ik) {
      const double ja = a[int64_t(ik) * nr], jb = b[int64_t(ik) * nr];
      const double2 kp = Kprod[ik];
      const double2 f = make_double2(kp.x * ja * jb, kp.y * ja * jb);
      const double dk = K[ik] - K[ik - 1];
      acc.x += dk * (flow.x + f.x);
      acc.y += dk * (flow.y + f.y);
      flow = f;
    }
    out[o] = acc;
  }
}

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ void block_partial(double v, double* __restrict__ partial) {
  __shared__ double red[kCollWarps];
  v = warp_sum(v);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < kCollWarps; ++w) s += red[w];
    partial[blockIdx.x] = s;
  }
}

template <int KT>
__global__ void __launch_bounds__(32 * kCollWarps)
coll_diag_kernel(const double2* __restrict__ A, const double2* __restrict__ B, int nlam, const int* __restrict__ rowL,
                 const int* __restrict__ rowM, int nrow, int Lmin, int Lmax, const double2* __restrict__ F, int nLF,
                 const double* __restrict__ w, int nr, double2 pref, double* __restrict__ partial) {
  const int lane = threadIdx.x & 31;
  const int64_t gw = int64_t(blockIdx.x) * kCollWarps + (threadIdx.x >> 5);
  const int64_t nw = int64_t(gridDim.x) * kCollWarps;
  double acc = 0.0;
  for (int64_t i = gw; i < nrow; i += nw) {
    const int L = rowL[i];
    if (L < Lmin || L > Lmax || L >= nLF) continue;
    const double mw = rowM[i] == 0 ? 1.0 : 2.0;
    const double2* FL = F + int64_t(L) * nr * nr;
    double2 x = make_double2(0.0, 0.0);  // Sum_lam Sum_k conj(B_k) w_k v_k of this lane's k
    for (int lam = 0; lam < nlam; ++lam) {
      const double2* a = A + (int64_t(lam) * nrow + i) * nr;
      const double2* b = B + (int64_t(lam) * nrow + i) * nr;
#pragma unroll
      for (int kt = 0; kt < KT; ++kt) {
        const int k = lane + 32 * kt;
        if (k >= nr) continue;
        double2 v = make_double2(0.0, 0.0);
        for (int j = 0; j < nr; ++j) v = cadd(v, cscale(cmul(a[j], FL[int64_t(j) * nr + k]), w[j]));
        x = cadd(x, cscale(cmul(v, cconj(b[k])), w[k]));
      }
    }
    acc += mw * (pref.x * x.x - pref.y * x.y);
  }
  block_partial(acc, partial);
}

__device__ __forceinline__ int lm_row_index(int Lp, int Mp, int nLmin, int nLmax) {
  const int am = abs(Mp);
  if (am > nLmin) return am * (nLmax - nLmin + 1) + (Lp - nLmin) - (am - nLmin) * (am - nLmin + 1) / 2;
  return am * (nLmax - nLmin + 1) + (Lp - nLmin);
}

// i^d for integer d
__device__ __forceinline__ double2 ipow(int d) {
  switch (((d % 4) + 4) % 4) {
    case 0: return make_double2(1.0, 0.0);
    case 1: return make_double2(0.0, 1.0);
    case 2: return make_double2(-1.0, 0.0);
    default: return make_double2(0.0, -1.0);
  }
}

template <int KT>
__global__ void __launch_bounds__(32 * kCollWarps)
coll_general_kernel(const double2* __restrict__ A1, const double2* __restrict__ A1c, const double2* __restrict__ A2,
                    const double2* __restrict__ A2c, const int* __restrict__ rowL, const int* __restrict__ rowM,
                    int nrow, int nLmin, int nLmax, int Lmin, int Lmax, const double2* __restrict__ F, int nLF, int nF,
                    const double* __restrict__ w, int nr, int s, int real_beta, const double2* __restrict__ coeffs,
                    double* __restrict__ partial) {
  const int lane = threadIdx.x & 31;
  const int64_t gw = int64_t(blockIdx.x) * kCollWarps + (threadIdx.x >> 5);
  const int64_t nw = int64_t(gridDim.x) * kCollWarps;
  double acc = 0.0;
  for (int64_t i = gw; i < nrow; i += nw) {
    const int L = rowL[i], M = rowM[i];
    if (L < Lmin || L > Lmax) continue;
    const int npiece = (!real_beta && M != 0) ? 2 : 1;
    for (int Delta = -2 * s; Delta <= 2 * s; ++Delta) {
      const int Lp = L + Delta;
      if (Lp < Lmin || Lp > Lmax || abs(Delta) > nF || L >= nLF) continue;
      const double2* FL = F + (int64_t(nF + Delta) * nLF + L) * nr * nr;
      for (int piece = 0; piece < npiece; ++piece) {
        for (int lam1 = -s; lam1 <= s; ++lam1) {
          // v_k = Sum_j A_j w_j F(r_j, r_k), A = arr1[s + lam1] (piece 0) or conj(arr1c[s - lam1]) (piece 1)
          const double2* a = piece == 0 ? A1 + (int64_t(s + lam1) * nrow + i) * nr
                                        : A1c + (int64_t(s - lam1) * nrow + i) * nr;
          double2 v[KT];
#pragma unroll
          for (int kt = 0; kt < KT; ++kt) {
            v[kt] = make_double2(0.0, 0.0);
            const int k = lane + 32 * kt;
            if (k >= nr) continue;
            for (int j = 0; j < nr; ++j) {
              const double2 aj = piece == 0 ? a[j] : cconj(a[j]);
              v[kt] = cadd(v[kt], cscale(cmul(aj, FL[int64_t(j) * nr + k]), w[j]));
            }
          }
          for (int S = 0; S <= 2 * s; S += 2) {
            if (abs(Delta) > S) continue;
            const double2 coeff = coeffs[S / 2];
            if (coeff.x == 0.0 && coeff.y == 0.0) continue;
            for (int Lam = -S; Lam <= S; ++Lam) {
              const int lam3 = -lam1 - Lam;
              if (abs(lam3) > s) continue;
              const int Mp = piece == 0 ? -M - Lam : M - Lam;
              if (abs(Mp) > Lp) continue;
              const double g = piece == 0 ? gaunt_small(L, Lp, S, M, Mp, Lam) : gaunt_small(L, Lp, S, -M, Mp, Lam);
              if (g == 0.0) continue;
              const double tj = threej_small(s, s, S, lam1, lam3, Lam);
              if (tj == 0.0) continue;
              double sg;
              if (piece == 0) {
                sg = (M != 0 && real_beta) ? 2.0 : 1.0;
                if (Mp < 0 && ((Mp + s + lam3) & 1)) sg = -sg;
              } else {
                sg = (Mp < 0) ? (((M + Mp + lam1 + lam3) & 1) ? -1.0 : 1.0) : (((s + lam1 + M) & 1) ? -1.0 : 1.0);
              }
              const double2 pref = cscale(cmul(coeff, ipow(Delta)), g * tj * sg);
              const int lmp = lm_row_index(Lp, Mp, nLmin, nLmax);
              const double2* b = Mp >= 0 ? A2 + (int64_t(s + lam3) * nrow + lmp) * nr
                                         : A2c + (int64_t(s - lam3) * nrow + lmp) * nr;
              double2 x = make_double2(0.0, 0.0);
#pragma unroll
              for (int kt = 0; kt < KT; ++kt) {
                const int k = lane + 32 * kt;
                if (k >= nr) continue;
                const double2 bk = Mp >= 0 ? b[k] : cconj(b[k]);
                x = cadd(x, cscale(cmul(bk, v[kt]), w[k]));
              }
              acc += pref.x * x.x - pref.y * x.y;
            }
          }
        }
      }
    }
  }
  block_partial(acc, partial);
}

template <int KT>
__global__ void __launch_bounds__(32 * kCollWarps)
coll_conv_kernel(const double2* __restrict__ PQ, const double2* __restrict__ cPQ, const int* __restrict__ rowL,
                 const int* __restrict__ rowM, const int* __restrict__ full_of_row, int nrow, int nLmin, int nLmax,
                 int Lmin, int Lmax, const double2* __restrict__ F, int nLF, int nrF, int nF,
                 const double* __restrict__ w, const int* __restrict__ inds, int nr, int s, int lam1,
                 const double2* __restrict__ Sw, double2* __restrict__ out_re, double2* __restrict__ out_im) {
  const int lane = threadIdx.x & 31;
  const int64_t gw = int64_t(blockIdx.x) * kCollWarps + (threadIdx.x >> 5);
  const int64_t nw = int64_t(gridDim.x) * kCollWarps;
  const double inv = 1.0 / (sqrt(2.0 * s + 1.0) * sqrt(4.0 * M_PI) * 2.0);
  for (int64_t i = gw; i < nrow; i += nw) {
    const int L = rowL[i], M = rowM[i];
    if (L < Lmin || L > Lmax || L >= nLF) continue;
    double2 plus[KT], minus[KT];
#pragma unroll
    for (int kt = 0; kt < KT; ++kt) plus[kt] = minus[kt] = make_double2(0.0, 0.0);
    // S = 0: diagonal in (L, M)
    const double2 S0 = Sw[0];
    if (S0.x != 0.0 || S0.y != 0.0) {
      const double2 pref = cscale(S0, (((s - lam1) & 1) ? -inv : inv) * (M == 0 ? 2.0 : 1.0));
      const double2 pref_m = cscale(cconj(S0), inv);
      const double2* a = PQ + (int64_t(s - lam1) * nrow + i) * nr;
      const double2* c = cPQ + (int64_t(s + lam1) * nrow + i) * nr;
      const double2* FL = F + (int64_t(nF) * nLF + L) * nrF * nrF;
#pragma unroll
      for (int kt = 0; kt < KT; ++kt) {
        const int j = lane + 32 * kt;
        if (j >= nr) continue;
        const double2* Fj = FL + int64_t(inds[j]) * nrF;
        double2 tp = make_double2(0.0, 0.0), tm = make_double2(0.0, 0.0);
        for (int k = 0; k < nr; ++k) {
          const double wk = w[k];
          if (wk == 0.0) continue;
          const double2 f = Fj[inds[k]];
          tp = cadd(tp, cscale(cmul(a[k], f), wk));
          if (M != 0) tm = cadd(tm, cscale(cmul(c[k], cconj(f)), wk));
        }
        plus[kt] = cadd(plus[kt], cmul(tp, pref));
        if (M != 0) minus[kt] = cadd(minus[kt], cmul(tm, pref_m));
      }
    }
    // S > 0
    for (int S = 2; S <= 2 * s; S += 2) {
      const double2 SwS = Sw[S / 2];
      for (int Delta = -S; Delta <= S; Delta += 2) {
        const int Lp = L + Delta;
        if (Lp < Lmin || Lp > Lmax || abs(Delta) > nF) continue;
        const double2* FL = F + (int64_t(nF + Delta) * nLF + L) * nrF * nrF;
        for (int lam = -S; lam <= S; ++lam) {
          const int lam3 = -lam1 - lam;
          if (abs(lam3) > s) continue;
          const double tj = threej_small(s, s, S, lam1, lam3, lam);
          const double2 pref = cscale(cmul(SwS, ipow(Delta)), tj);
          if (pref.x == 0.0 && pref.y == 0.0) continue;
          for (int part = 0; part < 2; ++part) {
            if (part == 1 && M == 0) break;
            const int Mp = part == 0 ? M - lam : -M - lam;
            if (abs(Mp) > Lp) continue;
            const double g = part == 0 ? gaunt_small(L, Lp, S, -M, M - lam, lam) : gaunt_small(L, Lp, S, M, -M - lam, lam);
            double sg;
            if (part == 0) sg = Mp >= 0 ? ((M & 1) ? -1.0 : 1.0) : (((M + Mp + s + lam3) & 1) ? -1.0 : 1.0);
            else sg = Mp >= 0 ? 1.0 : (((Mp + s + lam3) & 1) ? -1.0 : 1.0);
            if (part == 1 || M != 0) sg *= 0.5;
            const double2 gaunt = cscale(part == 0 ? pref : cconj(pref), g * sg);
            if (gaunt.x == 0.0 && gaunt.y == 0.0) continue;
            const int lmp = lm_row_index(Lp, Mp, nLmin, nLmax);
            const double2* b = Mp >= 0 ? PQ + (int64_t(s + lam3) * nrow + lmp) * nr
                                       : cPQ + (int64_t(s - lam3) * nrow + lmp) * nr;
#pragma unroll
            for (int kt = 0; kt < KT; ++kt) {
              const int j = lane + 32 * kt;
              if (j >= nr) continue;
              const double2* Fj = FL + int64_t(inds[j]) * nrF;
              double2 ks = make_double2(0.0, 0.0);
              for (int k = 0; k < nr; ++k) {
                const double wk = w[k];
                if (wk == 0.0) continue;
                const double2 f = Fj[inds[k]];
                double2 v;
                if (part == 0) v = cmul(Mp >= 0 ? b[k] : cconj(b[k]), f);
                else v = cmul(Mp >= 0 ? cconj(b[k]) : b[k], cconj(f));
                ks = cadd(ks, cscale(v, wk));
              }
              if (part == 0) plus[kt] = cadd(plus[kt], cmul(ks, gaunt));
              else minus[kt] = cadd(minus[kt], cmul(ks, gaunt));
            }
          }
        }
      }
    }
    const int full = full_of_row[i];
    if (full < 0) continue;
#pragma unroll
    for (int kt = 0; kt < KT; ++kt) {
      const int j = lane + 32 * kt;
      if (j >= nr) continue;
      const int64_t o = int64_t(full) * nr + j;
      out_re[o] = cadd(out_re[o], cadd(plus[kt], minus[kt]));
      out_im[o] = cadd(out_im[o], csub(plus[kt], minus[kt]));
    }
  }
}

__global__ void pF_complex_kernel(const double2* __restrict__ plus, const double2* __restrict__ minus, int lmax_in,
                                  int nin, const double2* __restrict__ p, int lsize, int npol, int nrp,
                                  const double* __restrict__ w, const int* __restrict__ inds,
                                  const int* __restrict__ ls, const int* __restrict__ ms, int64_t nl, int n1, int mu1,
                                  int nmax, double2* __restrict__ out) {
  const int64_t total = nl * npol;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total; t += int64_t(gridDim.x) * blockDim.x) {
    const int64_t i = t % nl;
    const int u = int(t / nl);
    const int l = ls[i], m = ms[i];
    double2 acc = make_double2(0.0, 0.0);
    for (int Delta = -n1; Delta <= n1; Delta += 2) {
      const int lp = l + Delta;
      if (lp > lmax_in || lp < 0) continue;
      const double2* pp = p + ((int64_t(nmax + Delta) * lsize + l) * npol + u) * nrp;
      for (int part = 0; part < 2; ++part) {
        const int mp = part == 0 ? m - mu1 : -m - mu1;
        if (abs(mp) > lp) continue;
        const int64_t idx = int64_t(abs(mp)) * (lmax_in + 1) + lp - int64_t(abs(mp)) * (abs(mp) + 1) / 2;
        const double G = part == 0 ? gaunt_small(l, lp, n1, m, -mp, -mu1) : gaunt_small(l, lp, n1, -m, -mp, -mu1);
        if (G == 0.0) continue;
        double2 gp = part == 0 ? cscale(ipow(Delta), ((m & 1) ? -0.25 : 0.25) * G) : cscale(ipow(-Delta), 0.25 * G);
        double2 s = make_double2(0.0, 0.0);
        for (int j = 0; j < nin; ++j) {
          const double wj = w[j];
          if (wj == 0.0) continue;
          const double2 pj = pp[inds[j]];
          double2 v;
          if (part == 0) v = mp >= 0 ? cmul(plus[idx * nin + j], pj) : cmul(cconj(minus[idx * nin + j]), pj);
          else v = mp >= 0 ? cconj(cmul(plus[idx * nin + j], pj)) : cmul(minus[idx * nin + j], cconj(pj));
          s = cadd(s, cscale(v, wj));
        }
        // gm = gp (-1)^mp, and the minus branch of part 1 carries a further (-1)^mp
        if (mp < 0 && part == 0 && (mp & 1)) gp = cscale(gp, -1.0);
        acc = cadd(acc, cmul(gp, s));
      }
    }
    out[int64_t(u) * nl + i] = cadd(out[int64_t(u) * nl + i], acc);
  }
}

__global__ void coll_sum_partials(const double* __restrict__ partial, int64_t n, double* __restrict__ out) {
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

// CTAs of the per-row kernels: one per kCollWarps rows, at most 8 per SM of the current device; the
// workspace query and the launches size by this one function (one partial sum per CTA)
int64_t coll_grid(int64_t nrow) {
  const int64_t cap = int64_t(device_sms()) * 8;
  const int64_t g = (nrow + kCollWarps - 1) / kCollWarps;
  return g > cap ? cap : (g < 1 ? 1 : g);
}

}  // namespace
}  // namespace ps

using namespace ps;

extern "C" int ps_kint_collider_jlK(const double* table, const double* x, int64_t nx, int nl, const double* K, int nK,
                                    const double* r, int nr, double* jlK, cudaStream_t stream) {
  if (!table || !x || !K || !r || !jlK || nx < 2 || nl <= 0 || nK <= 0 || nr <= 0) return PS_ERR_INVALID;
  StatScope sc(PS_K_VECTOR, 0.0, 8.0 * double(nl) * nK * nr, stream);
  int64_t g = (int64_t(nK) * nr + 255) / 256;
  if (g > 148 * 16) g = 148 * 16;
  coll_jlK_kernel<<<int(g), 256, 0, stream>>>(table, x, nx, nl, K, nK, r, nr, jlK);
  PS_LAUNCH_CHECK();
  return PS_OK;
}

extern "C" int ps_kint_collider_F(const double* jlK, int nl_tab, int glmin, const double* K, int nK,
                                  const double* Kprod, int nr, int Lmin, int Lmax, int nmax_F, int nLout, double* out,
                                  cudaStream_t stream) {
  if (!jlK || !K || !Kprod || !out || nl_tab <= 0 || glmin < 0 || nK < 1 || nr <= 0 || Lmin < 0 || Lmax < Lmin ||
      nmax_F < 0 || nLout <= 0)
    return PS_ERR_INVALID;
  const int nL = Lmax + nmax_F - max(Lmin - nmax_F, 0) + 1;
  const int64_t total = int64_t(2 * nmax_F + 1) * nL * nr * nr;
  StatScope sc(PS_K_VECTOR, 0.0, 16.0 * double(total), stream);
  int64_t g = (total + 127) / 128;
  if (g > 148 * 32) g = 148 * 32;
  coll_F_kernel<<<int(g), 128, 0, stream>>>(jlK, nl_tab, glmin, K, nK, reinterpret_cast<const double2*>(Kprod), nr,
                                            Lmin, Lmax, nmax_F, nLout, reinterpret_cast<double2*>(out));
  PS_LAUNCH_CHECK();
  return PS_OK;
}

extern "C" int ps_tau_collider_workspace_bytes(int64_t nrow, size_t* bytes) {
  if (!bytes || nrow <= 0) return PS_ERR_INVALID;
  *bytes = sizeof(double) * size_t(coll_grid(nrow));
  return PS_OK;
}

extern "C" int ps_tau_sum_collider_diag(const double* A, const double* B, int nlam, const int* rowL, const int* rowM,
                                        int nrow, int Lmin, int Lmax, const double* F, int nLF, const double* w,
                                        int nr, double pref_re, double pref_im, double* out, void* workspace,
                                        size_t workspace_bytes, cudaStream_t stream) {
  if (!A || !B || !rowL || !rowM || !F || !w || !out || nlam <= 0 || nrow <= 0 || nr <= 0 || nr > 64 || nLF <= 0)
    return PS_ERR_INVALID;
  const int64_t nblk = coll_grid(nrow);
  if (!workspace || workspace_bytes < sizeof(double) * size_t(nblk)) return PS_ERR_WORKSPACE;
  StatScope sc(PS_K_PIXEL, 0.0, 16.0 * double(nrow) * nr * (2 * nlam + nr), stream);
  const double2 pref = make_double2(pref_re, pref_im);
  const double2* a = reinterpret_cast<const double2*>(A);
  const double2* b = reinterpret_cast<const double2*>(B);
  const double2* f = reinterpret_cast<const double2*>(F);
  double* part = static_cast<double*>(workspace);
  if (nr <= 32)
    coll_diag_kernel<1><<<unsigned(nblk), 32 * kCollWarps, 0, stream>>>(a, b, nlam, rowL, rowM, nrow, Lmin, Lmax, f,
                                                                       nLF, w, nr, pref, part);
  else
    coll_diag_kernel<2><<<unsigned(nblk), 32 * kCollWarps, 0, stream>>>(a, b, nlam, rowL, rowM, nrow, Lmin, Lmax, f,
                                                                       nLF, w, nr, pref, part);
  PS_LAUNCH_CHECK();
  coll_sum_partials<<<1, 256, 0, stream>>>(part, nblk, out);
  PS_LAUNCH_CHECK();
  return PS_OK;
}

extern "C" int ps_tau_sum_collider_general(const double* A1, const double* A1c, const double* A2, const double* A2c,
                                           const int* rowL, const int* rowM, int nrow, int nLmin, int nLmax, int Lmin,
                                           int Lmax, const double* F, int nLF, int nmax_F, const double* w, int nr,
                                           int s, int real_beta, const double* coeffs, double* out, void* workspace,
                                           size_t workspace_bytes, cudaStream_t stream) {
  if (!A1 || !A1c || !A2 || !A2c || !rowL || !rowM || !F || !w || !coeffs || !out || nrow <= 0 || nr <= 0 ||
      nr > 64 || s < 0 || s > 5 || nmax_F < 0 || nLF <= Lmax || nLmin < 0 || nLmax < nLmin || Lmin < nLmin ||
      Lmax > nLmax)
    return PS_ERR_INVALID;
  const int64_t nblk = coll_grid(nrow);
  if (!workspace || workspace_bytes < sizeof(double) * size_t(nblk)) return PS_ERR_WORKSPACE;
  StatScope sc(PS_K_PIXEL, 0.0, 16.0 * double(nrow) * nr * (4 * s + 1) * (2 * s + 1) * (nr + 2), stream);
  const double2* a1 = reinterpret_cast<const double2*>(A1);
  const double2* a1c = reinterpret_cast<const double2*>(A1c);
  const double2* a2 = reinterpret_cast<const double2*>(A2);
  const double2* a2c = reinterpret_cast<const double2*>(A2c);
  const double2* f = reinterpret_cast<const double2*>(F);
  const double2* c = reinterpret_cast<const double2*>(coeffs);
  double* part = static_cast<double*>(workspace);
  if (nr <= 32)
    coll_general_kernel<1><<<unsigned(nblk), 32 * kCollWarps, 0, stream>>>(
        a1, a1c, a2, a2c, rowL, rowM, nrow, nLmin, nLmax, Lmin, Lmax, f, nLF, nmax_F, w, nr, s, real_beta, c, part);
  else
    coll_general_kernel<2><<<unsigned(nblk), 32 * kCollWarps, 0, stream>>>(
        a1, a1c, a2, a2c, rowL, rowM, nrow, nLmin, nLmax, Lmin, Lmax, f, nLF, nmax_F, w, nr, s, real_beta, c, part);
  PS_LAUNCH_CHECK();
  coll_sum_partials<<<1, 256, 0, stream>>>(part, nblk, out);
  PS_LAUNCH_CHECK();
  return PS_OK;
}

extern "C" int ps_convolve_F_collider(const double* PQ, const double* cPQ, const int* rowL, const int* rowM,
                                      const int* full_of_row, int nrow, int nLmin, int nLmax, int Lmin, int Lmax,
                                      const double* F, int nLF, int nrF, int nmax_F, const double* w, const int* inds,
                                      int nr, int s, int lam1, const double* S_weights, double* out_re,
                                      double* out_im, cudaStream_t stream) {
  if (!PQ || !cPQ || !rowL || !rowM || !full_of_row || !F || !w || !inds || !S_weights || !out_re || !out_im ||
      nrow <= 0 || nr <= 0 || nr > 64 || nrF < nr || s < 0 || s > 5 || abs(lam1) > s || nmax_F < 0 || nLF <= Lmax ||
      nLmin < 0 || nLmax < nLmin || Lmin < nLmin || Lmax > nLmax)
    return PS_ERR_INVALID;
  StatScope sc(PS_K_PIXEL, 0.0, 16.0 * double(nrow) * nr * nr * (2 * s + 1) * (2 * s + 1), stream);
  const int64_t g = coll_grid(nrow);
  const double2* a = reinterpret_cast<const double2*>(PQ);
  const double2* c = reinterpret_cast<const double2*>(cPQ);
  const double2* f = reinterpret_cast<const double2*>(F);
  const double2* sw = reinterpret_cast<const double2*>(S_weights);
  double2* ore = reinterpret_cast<double2*>(out_re);
  double2* oim = reinterpret_cast<double2*>(out_im);
  if (nr <= 32)
    coll_conv_kernel<1><<<unsigned(g), 32 * kCollWarps, 0, stream>>>(a, c, rowL, rowM, full_of_row, nrow, nLmin,
                                                                    nLmax, Lmin, Lmax, f, nLF, nrF, nmax_F, w, inds,
                                                                    nr, s, lam1, sw, ore, oim);
  else
    coll_conv_kernel<2><<<unsigned(g), 32 * kCollWarps, 0, stream>>>(a, c, rowL, rowM, full_of_row, nrow, nLmin,
                                                                    nLmax, Lmin, Lmax, f, nLF, nrF, nmax_F, w, inds,
                                                                    nr, s, lam1, sw, ore, oim);
  PS_LAUNCH_CHECK();
  return PS_OK;
}

extern "C" int ps_pF_map_complex(const double* plus, const double* minus, int lmax_in, int nin, const double* p,
                                 int nshift, int lsize, int npol, int nrp, const double* w, const int* inds,
                                 const int* ls, const int* ms, int64_t nl, int n1, int mu1, int nmax, double* out,
                                 cudaStream_t stream) {
  if (!plus || !minus || !p || !w || !inds || !ls || !ms || !out || lmax_in < 0 || nin <= 0 || nshift != 2 * nmax + 1 ||
      n1 < 0 || n1 > 16 || n1 > nmax || abs(mu1) > n1 || npol <= 0 || nl <= 0 || nrp <= 0)
    return PS_ERR_INVALID;
  StatScope sc(PS_K_PIXEL, 0.0, 16.0 * double(nl) * npol * nin * (n1 + 1) * 2, stream);
  int64_t g = (nl * npol + 127) / 128;
  if (g > 148 * 64) g = 148 * 64;
  pF_complex_kernel<<<int(g), 128, 0, stream>>>(reinterpret_cast<const double2*>(plus),
                                                reinterpret_cast<const double2*>(minus), lmax_in, nin,
                                                reinterpret_cast<const double2*>(p), lsize, npol, nrp, w, inds, ls, ms,
                                                nl, n1, mu1, nmax, reinterpret_cast<double2*>(out));
  PS_LAUNCH_CHECK();
  return PS_OK;
}
