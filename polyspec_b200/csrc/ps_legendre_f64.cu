// FP64 Legendre stage of the HEALPix SHT (the plain-precision backend).
//
// Synthesis, per order m and ring pair (theta, pi - theta):
//   spin 0:  F_m(theta) = sum_l lam_lm(theta) a_lm, split by the parity of l+m
//            so that the mirror ring is  E - O  where the north ring is E + O.
//   spin s:  the same with F+ = (+s lam + -s lam)/2 and F- = (+s lam - -s lam)/2
//            against G and C (HEALPix conventions of polyspec/base.py:247-288).
// Adjoint: a_lm = sum_rings lam_lm(theta_r) P_m(r) (and the spin analogue),
// the exact adjoint under the m-weighted alm inner product of
// polyspec/weighting.py:255, i.e. ducc0.sht.adjoint_synthesis.
//
// The recurrences (normalised associated Legendre functions for spin 0,
// spin-weighted harmonics in the Goldberg/HEALPix convention for spin s) run in
// FP64 with seeds scaled by 2^(800k) so that high m near the poles neither
// underflows nor loses accuracy (Reinecke & Seljebotn 2013).
//
// Layouts: almT [nalm][B][ncomp] (m-major l within, map index and G/C
// innermost), phase [R][mmax+1][B][ncomp] (ring-major, order m, then maps).
#include "ps_common.cuh"
#include "ps_stats.cuh"

namespace ps {

constexpr int SYN_THREADS = 128;  // ring pairs per synthesis CTA
constexpr int SYN_LCH = 64;       // l chunk staged in shared memory
constexpr int ADJ_THREADS = 128;  // ring pairs per adjoint CTA (== ring tile)
constexpr int ADJ_LCH = 16;       // l chunk of the adjoint's Legendre tile

// ---------------------------------------------------------------- seeds
__device__ __forceinline__ void seed_spin0(int m, double sth, double mnorm, double& v, int& k) {
  Scaled s = smul(spow(sth, m), snorm(mnorm));
  to_kscale(s, v, k);
  if (m & 1) v = -v;
}

// Seeds of +s lam and -s lam at l = max(m, s) (Goldberg et al. 1967 with a
// single term left in the sum), with a common scale exponent k.
__device__ __forceinline__ void seed_spin(int m, int s, const RingInfo& g, SeedNorm nrm, double& f, double& gg,
                                          int& k) {
  const double sh = sqrt(0.5 * g.omz), ch = sqrt(0.5 * g.opz);
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
  Scaled n; n.v = nrm.v; n.e = nrm.e;
  Scaled sf = smul(n, pf), sg = smul(n, pg);
  Scaled big = (sf.e >= sg.e) ? sf : sg;
  double vb;
  to_kscale(big, vb, k);
  const int shift = k * SCALE_BITS;
  f = ldexp(sf.v, max(sf.e - shift, -2000)) * sgn_f;
  gg = ldexp(sg.v, max(sg.e - shift, -2000)) * sgn_g;
}

// spin-0 recurrence coefficients to step lam_{l-1} -> lam_l:
//   lam_l = a_l x lam_{l-1} - b_l lam_{l-2},  a_l = sqrt((4l^2-1)/(l^2-m^2)), b_l = a_l/a_{l-1}
__device__ __forceinline__ void coef_spin0(int l, int m, double& a, double& b) {
  const double mm = double(m) * m;
  a = sqrt((4.0 * l * l - 1.0) / (double(l) * l - mm));
  b = 0.0;
  if (l >= m + 2) b = a / sqrt((4.0 * (l - 1.0) * (l - 1.0) - 1.0) / ((l - 1.0) * (l - 1.0) - mm));
}

// spin-s coefficients to step l -> l+1 (l >= max(m, s)):
//   f_{l+1} = (A x + D) f_l - C f_{l-1},  g_{l+1} = (A x - D) g_l - C g_{l-1}
__device__ __forceinline__ void coef_spin(int l, int m, int s, double& A, double& D, double& C) {
  auto rho = [&](double L) {
    return sqrt(fmax(L * L - double(m) * m, 0.0) * fmax(L * L - double(s) * s, 0.0));
  };
  const double r1 = rho(l + 1.0), q = sqrt((2.0 * l + 3.0) * (2.0 * l + 1.0));
  A = q * (l + 1.0) / r1;
  D = q * double(m) * double(s) / (double(l) * r1);
  C = sqrt((2.0 * l + 3.0) / (2.0 * l - 1.0)) * (l + 1.0) * rho(double(l)) / (double(l) * r1);
}

// =====================================================================
// synthesis, spin 0
// grid (ceil(Rh/SYN_THREADS), mmax+1, ceil(B/NB))
template <int NB>
__global__ void __launch_bounds__(SYN_THREADS) synth0_f64(const RingInfo* __restrict__ rings,
                                                           const double* __restrict__ mnorm,
                                                           const double2* __restrict__ almT,
                                                           double2* __restrict__ phase, int R, int Rh, int lmax,
                                                           int mmax, int B) {
  const int m = blockIdx.y;
  const int rp = blockIdx.x * SYN_THREADS + threadIdx.x;
  const int b0 = blockIdx.z * NB;
  __shared__ double s_a[SYN_LCH], s_b[SYN_LCH];
  __shared__ double2 s_alm[SYN_LCH][NB];
  const bool active = rp < Rh;
  const RingInfo g = rings[active ? rp : 0];
  const double x = g.z;
  double cur, prev = 0.0;
  int k;
  seed_spin0(m, g.sth, mnorm[m], cur, k);
  double2 ae[NB], ao[NB];
#pragma unroll
  for (int i = 0; i < NB; ++i) { ae[i] = make_double2(0.0, 0.0); ao[i] = ae[i]; }
  const int64_t base = alm_index(m, m, lmax);
  for (int l0 = m; l0 <= lmax; l0 += SYN_LCH) {
    const int n = min(SYN_LCH, lmax - l0 + 1);
    for (int j = threadIdx.x; j < SYN_LCH; j += SYN_THREADS) {
      double a = 0.0, b = 0.0;
      const int l = l0 + j + 1;  // coefficients producing lam_{l0+j+1}
      if (l <= lmax) coef_spin0(l, m, a, b);
      s_a[j] = a; s_b[j] = b;
    }
    for (int t = threadIdx.x; t < n * NB; t += SYN_THREADS) {
      const int j = t / NB, bi = t % NB;
      s_alm[j][bi] = (b0 + bi < B) ? almT[(base + (l0 - m) + j) * B + b0 + bi] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    // l0 + m is even, so even j are parity 0 and odd j parity 1
    auto step = [&](int j, double2* acc) {
      const double val = (k == 0) ? cur : 0.0;
#pragma unroll
      for (int i = 0; i < NB; ++i) acc[i] = cfma(val, s_alm[j][i], acc[i]);
      const double nxt = s_a[j] * x * cur - s_b[j] * prev;
      prev = cur;
      cur = nxt;
      if (k < 0 && fabs(cur) > PS_FTHRESH) { cur *= PS_FSMALL; prev *= PS_FSMALL; ++k; }
    };
    int j = 0;
    for (; j + 1 < n; j += 2) { step(j, ae); step(j + 1, ao); }
    if (j < n) step(j, ae);
    __syncthreads();
  }
  if (!active) return;
  const int rs = R - 1 - rp;
#pragma unroll
  for (int i = 0; i < NB; ++i) {
    if (b0 + i >= B) break;
    phase[(int64_t(rp) * (mmax + 1) + m) * B + b0 + i] = cadd(ae[i], ao[i]);
    if (rs != rp) phase[(int64_t(rs) * (mmax + 1) + m) * B + b0 + i] = csub(ae[i], ao[i]);
  }
}

// =====================================================================
// synthesis, spin s > 0.  almT [nalm][B][2] (G,C); phase [R][mmax+1][B][2] (Q,U)
template <int NB>
__global__ void __launch_bounds__(SYN_THREADS) synthS_f64(const RingInfo* __restrict__ rings,
                                                           const SeedNorm* __restrict__ seednorm,
                                                           const double2* __restrict__ almT,
                                                           double2* __restrict__ phase, int R, int Rh, int lmax,
                                                           int mmax, int B, int spin) {
  const int m = blockIdx.y;
  const int rp = blockIdx.x * SYN_THREADS + threadIdx.x;
  const int b0 = blockIdx.z * NB;
  __shared__ double s_A[SYN_LCH], s_D[SYN_LCH], s_C[SYN_LCH];
  __shared__ double2 s_alm[SYN_LCH][NB][2];
  const bool active = rp < Rh;
  const RingInfo g = rings[active ? rp : 0];
  const double x = g.z;
  const int lmin = max(m, spin);
  double sf, sg;
  int k;
  seed_spin(m, spin, g, seednorm[m], sf, sg, k);
  double f = 0.0, gg = 0.0, fp = 0.0, gp = 0.0;
  // accumulators [parity]: G*F+, G*F-, C*F+, C*F-
  double2 GP[2][NB], GM[2][NB], CP[2][NB], CM[2][NB];
#pragma unroll
  for (int p = 0; p < 2; ++p)
#pragma unroll
    for (int i = 0; i < NB; ++i) {
      GP[p][i] = make_double2(0.0, 0.0); GM[p][i] = GP[p][i]; CP[p][i] = GP[p][i]; CM[p][i] = GP[p][i];
    }
  const int64_t base = alm_index(m, m, lmax);
  for (int l0 = m; l0 <= lmax; l0 += SYN_LCH) {
    const int n = min(SYN_LCH, lmax - l0 + 1);
    for (int j = threadIdx.x; j < SYN_LCH; j += SYN_THREADS) {
      double A = 0.0, D = 0.0, C = 0.0;
      const int l = l0 + j;  // step l -> l+1
      if (l >= lmin && l < lmax) coef_spin(l, m, spin, A, D, C);
      s_A[j] = A; s_D[j] = D; s_C[j] = C;
    }
    for (int t = threadIdx.x; t < n * NB; t += SYN_THREADS) {
      const int j = t / NB, bi = t % NB;
      const bool ok = b0 + bi < B;
      const int64_t idx = ((base + (l0 - m) + j) * B + b0 + bi) * 2;
      s_alm[j][bi][0] = ok ? almT[idx] : make_double2(0.0, 0.0);
      s_alm[j][bi][1] = ok ? almT[idx + 1] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    auto step = [&](int j, int p) {
      const int l = l0 + j;
      if (l == lmin) { f = sf; gg = sg; fp = 0.0; gp = 0.0; }
      const double vf = (k == 0) ? 0.5 * (f + gg) : 0.0;  // F+
      const double vm = (k == 0) ? 0.5 * (f - gg) : 0.0;  // F-
#pragma unroll
      for (int i = 0; i < NB; ++i) {
        const double2 G = s_alm[j][i][0], C = s_alm[j][i][1];
        GP[p][i] = cfma(vf, G, GP[p][i]);
        GM[p][i] = cfma(vm, G, GM[p][i]);
        CP[p][i] = cfma(vf, C, CP[p][i]);
        CM[p][i] = cfma(vm, C, CM[p][i]);
      }
      const double ax = s_A[j] * x;
      const double fn = (ax + s_D[j]) * f - s_C[j] * fp;
      const double gn = (ax - s_D[j]) * gg - s_C[j] * gp;
      fp = f; f = fn; gp = gg; gg = gn;
      if (k < 0 && fmax(fabs(f), fabs(gg)) > PS_FTHRESH) {
        f *= PS_FSMALL; fp *= PS_FSMALL; gg *= PS_FSMALL; gp *= PS_FSMALL; ++k;
      }
    };
    int j = 0;
    for (; j + 1 < n; j += 2) { step(j, 0); step(j + 1, 1); }
    if (j < n) step(j, 0);
    __syncthreads();
  }
  if (!active) return;
  const int rs = R - 1 - rp;
  const bool odd = spin & 1;
#pragma unroll
  for (int i = 0; i < NB; ++i) {
    if (b0 + i >= B) break;
    for (int side = 0; side < (rs != rp ? 2 : 1); ++side) {
      // north: F+ and F- sums add; south: F+ -> (-1)^p, F- -> -(-1)^p
      const double2 gps = side == 0 ? cadd(GP[0][i], GP[1][i]) : csub(GP[0][i], GP[1][i]);
      const double2 gms = side == 0 ? cadd(GM[0][i], GM[1][i]) : csub(GM[1][i], GM[0][i]);
      const double2 cps = side == 0 ? cadd(CP[0][i], CP[1][i]) : csub(CP[0][i], CP[1][i]);
      const double2 cms = side == 0 ? cadd(CM[0][i], CM[1][i]) : csub(CM[1][i], CM[0][i]);
      double2 q, u;
      if (!odd) {  // Q = -(G F+ + i C F-),  U = i G F- - C F+
        q = make_double2(-(gps.x - cms.y), -(gps.y + cms.x));
        u = make_double2(-gms.y - cps.x, gms.x - cps.y);
      } else {     // Q = -(G F- + i C F+),  U = i G F+ - C F-
        q = make_double2(-(gms.x - cps.y), -(gms.y + cps.x));
        u = make_double2(-gps.y - cms.x, gps.x - cms.y);
      }
      const int rr = side == 0 ? rp : rs;
      const int64_t o = ((int64_t(rr) * (mmax + 1) + m) * B + b0 + i) * 2;
      phase[o] = q;
      phase[o + 1] = u;
    }
  }
}

// =====================================================================
// adjoint, spin 0.  One CTA per (ring tile of ADJ_THREADS pairs, m, map chunk):
// the tile's threads run the recurrence of their ring and drop lam into a
// shared [ADJ_LCH][ADJ_THREADS] tile; then each thread reduces one l over a
// strided subset of rings and the 8 subsets of a warp are combined by
// shuffles.  Output: partial[tile][nalm][B] (summed by reduce_partials).
//
// reduction mapping (4 warps): warp w -> parity p = w & 1, jset = w >> 1;
// lane -> jq = lane >> 3, seg = lane & 7; l offset j = p + 2 (4 jset + jq);
// rings seg, seg+8, ..., seg+120.
template <int NB>
__global__ void __launch_bounds__(ADJ_THREADS) adj0_f64(const RingInfo* __restrict__ rings,
                                                         const double* __restrict__ mnorm,
                                                         const double2* __restrict__ phase,
                                                         double2* __restrict__ partial, int R, int Rh, int lmax,
                                                         int mmax, int B, int bofs, int Bc, int64_t nalm) {
  const int m = blockIdx.y;
  const int tile = blockIdx.x;
  const int tid = threadIdx.x;
  const int rp = tile * ADJ_THREADS + tid;
  const int b0 = bofs + blockIdx.z * NB;
  // ring-contiguous layouts (a warp's 8 ring segments read consecutive words)
  __shared__ double s_lam[ADJ_LCH][ADJ_THREADS + 2];
  __shared__ double2 s_P[2][NB][ADJ_THREADS];  // [even/odd][map][ring]
  __shared__ double s_a[ADJ_LCH], s_b[ADJ_LCH];
  const bool active = rp < Rh;
  const RingInfo g = rings[active ? rp : 0];
  const int rs = R - 1 - rp;
#pragma unroll
  for (int i = 0; i < NB; ++i) {
    double2 pn = make_double2(0.0, 0.0), ps = pn;
    if (active && b0 + i < bofs + Bc) {
      pn = phase[(int64_t(rp) * (mmax + 1) + m) * B + b0 + i];
      if (rs != rp) ps = phase[(int64_t(rs) * (mmax + 1) + m) * B + b0 + i];
    }
    s_P[0][i][tid] = cadd(pn, ps);
    s_P[1][i][tid] = csub(pn, ps);
  }
  const double x = g.z;
  double cur, prev = 0.0;
  int k;
  seed_spin0(m, g.sth, mnorm[m], cur, k);
  if (!active) { cur = 0.0; k = 0; }
  const int warp = tid >> 5, lane = tid & 31;
  const int p = warp & 1, jset = warp >> 1, jq = lane >> 3, seg = lane & 7;
  const int jr = p + 2 * (4 * jset + jq);
  const int64_t base = alm_index(m, m, lmax);
  for (int l0 = m; l0 <= lmax; l0 += ADJ_LCH) {
    const int n = min(ADJ_LCH, lmax - l0 + 1);
    if (tid < ADJ_LCH) {
      double a = 0.0, b = 0.0;
      const int l = l0 + tid + 1;
      if (l <= lmax) coef_spin0(l, m, a, b);
      s_a[tid] = a; s_b[tid] = b;
    }
    __syncthreads();
    for (int j = 0; j < ADJ_LCH; ++j) {
      s_lam[j][tid] = (k == 0) ? cur : 0.0;
      const double nxt = s_a[j] * x * cur - s_b[j] * prev;
      prev = cur;
      cur = nxt;
      if (k < 0 && fabs(cur) > PS_FTHRESH) { cur *= PS_FSMALL; prev *= PS_FSMALL; ++k; }
    }
    __syncthreads();
    double2 acc[NB];
#pragma unroll
    for (int i = 0; i < NB; ++i) acc[i] = make_double2(0.0, 0.0);
#pragma unroll 4
    for (int t = 0; t < ADJ_THREADS / 8; ++t) {
      const int r = seg + 8 * t;
      const double lam = s_lam[jr][r];
#pragma unroll
      for (int i = 0; i < NB; ++i) acc[i] = cfma(lam, s_P[p][i][r], acc[i]);
    }
#pragma unroll
    for (int i = 0; i < NB; ++i) {
#pragma unroll
      for (int off = 1; off < 8; off <<= 1) {
        acc[i].x += __shfl_xor_sync(0xffffffffu, acc[i].x, off);
        acc[i].y += __shfl_xor_sync(0xffffffffu, acc[i].y, off);
      }
    }
    if (seg == 0 && jr < n) {
      const int64_t idx = base + (l0 - m) + jr;
#pragma unroll
      for (int i = 0; i < NB; ++i)
        if (b0 + i < bofs + Bc) partial[(int64_t(tile) * nalm + idx) * Bc + (b0 - bofs) + i] = acc[i];
    }
    __syncthreads();
  }
}

// =====================================================================
// adjoint, spin s.  phase [R][mmax+1][B][2] (Q,U) -> partial[tile][nalm][B][2] (G,C)
template <int NB>
__global__ void __launch_bounds__(ADJ_THREADS) adjS_f64(const RingInfo* __restrict__ rings,
                                                         const SeedNorm* __restrict__ seednorm,
                                                         const double2* __restrict__ phase,
                                                         double2* __restrict__ partial, int R, int Rh, int lmax,
                                                         int mmax, int B, int bofs, int Bc, int64_t nalm, int spin) {
  const int m = blockIdx.y;
  const int tile = blockIdx.x;
  const int tid = threadIdx.x;
  const int rp = tile * ADJ_THREADS + tid;
  const int b0 = bofs + blockIdx.z * NB;
  __shared__ double s_fp[ADJ_LCH][ADJ_THREADS + 2];
  __shared__ double s_fm[ADJ_LCH][ADJ_THREADS + 2];
  __shared__ double2 s_Q[2][NB][ADJ_THREADS];  // [N+S, N-S][map][ring]
  __shared__ double2 s_U[2][NB][ADJ_THREADS];
  __shared__ double s_A[ADJ_LCH], s_D[ADJ_LCH], s_C[ADJ_LCH];
  const bool active = rp < Rh;
  const RingInfo g = rings[active ? rp : 0];
  const int rs = R - 1 - rp;
#pragma unroll
  for (int i = 0; i < NB; ++i) {
    double2 qn = make_double2(0.0, 0.0), qs = qn, un = qn, us = qn;
    if (active && b0 + i < bofs + Bc) {
      const int64_t o = ((int64_t(rp) * (mmax + 1) + m) * B + b0 + i) * 2;
      qn = phase[o]; un = phase[o + 1];
      if (rs != rp) {
        const int64_t o2 = ((int64_t(rs) * (mmax + 1) + m) * B + b0 + i) * 2;
        qs = phase[o2]; us = phase[o2 + 1];
      }
    }
    s_Q[0][i][tid] = cadd(qn, qs); s_Q[1][i][tid] = csub(qn, qs);
    s_U[0][i][tid] = cadd(un, us); s_U[1][i][tid] = csub(un, us);
  }
  const double x = g.z;
  const int lmin = max(m, spin);
  double sf, sg;
  int k;
  seed_spin(m, spin, g, seednorm[m], sf, sg, k);
  if (!active) { sf = 0.0; sg = 0.0; k = 0; }
  double f = 0.0, gg = 0.0, fpv = 0.0, gpv = 0.0;
  const int warp = tid >> 5, lane = tid & 31;
  const int p = warp & 1, jset = warp >> 1, jq = lane >> 3, seg = lane & 7;
  const int jr = p + 2 * (4 * jset + jq);
  // F+ multiplies (N + (-1)^p S), F- multiplies (N - (-1)^p S)
  const int cplus = p, cminus = 1 - p;
  const bool odd = spin & 1;
  const int64_t base = alm_index(m, m, lmax);
  for (int l0 = m; l0 <= lmax; l0 += ADJ_LCH) {
    const int n = min(ADJ_LCH, lmax - l0 + 1);
    if (tid < ADJ_LCH) {
      double A = 0.0, D = 0.0, C = 0.0;
      const int l = l0 + tid;
      if (l >= lmin && l < lmax) coef_spin(l, m, spin, A, D, C);
      s_A[tid] = A; s_D[tid] = D; s_C[tid] = C;
    }
    __syncthreads();
    for (int j = 0; j < ADJ_LCH; ++j) {
      if (l0 + j == lmin) { f = sf; gg = sg; fpv = 0.0; gpv = 0.0; }
      s_fp[j][tid] = (k == 0) ? 0.5 * (f + gg) : 0.0;
      s_fm[j][tid] = (k == 0) ? 0.5 * (f - gg) : 0.0;
      const double ax = s_A[j] * x;
      const double fn = (ax + s_D[j]) * f - s_C[j] * fpv;
      const double gn = (ax - s_D[j]) * gg - s_C[j] * gpv;
      fpv = f; f = fn; gpv = gg; gg = gn;
      if (k < 0 && fmax(fabs(f), fabs(gg)) > PS_FTHRESH) {
        f *= PS_FSMALL; fpv *= PS_FSMALL; gg *= PS_FSMALL; gpv *= PS_FSMALL; ++k;
      }
    }
    __syncthreads();
    // S1 = sum F+ Q+, S2 = sum F- U-, S3 = sum F- Q-, S4 = sum F+ U+
    double2 S1[NB], S2[NB], S3[NB], S4[NB];
#pragma unroll
    for (int i = 0; i < NB; ++i) {
      S1[i] = make_double2(0.0, 0.0); S2[i] = S1[i]; S3[i] = S1[i]; S4[i] = S1[i];
    }
#pragma unroll 2
    for (int t = 0; t < ADJ_THREADS / 8; ++t) {
      const int r = seg + 8 * t;
      const double vp = s_fp[jr][r], vm = s_fm[jr][r];
#pragma unroll
      for (int i = 0; i < NB; ++i) {
        S1[i] = cfma(vp, s_Q[cplus][i][r], S1[i]);
        S2[i] = cfma(vm, s_U[cminus][i][r], S2[i]);
        S3[i] = cfma(vm, s_Q[cminus][i][r], S3[i]);
        S4[i] = cfma(vp, s_U[cplus][i][r], S4[i]);
      }
    }
#pragma unroll
    for (int i = 0; i < NB; ++i) {
#pragma unroll
      for (int off = 1; off < 8; off <<= 1) {
        S1[i].x += __shfl_xor_sync(0xffffffffu, S1[i].x, off); S1[i].y += __shfl_xor_sync(0xffffffffu, S1[i].y, off);
        S2[i].x += __shfl_xor_sync(0xffffffffu, S2[i].x, off); S2[i].y += __shfl_xor_sync(0xffffffffu, S2[i].y, off);
        S3[i].x += __shfl_xor_sync(0xffffffffu, S3[i].x, off); S3[i].y += __shfl_xor_sync(0xffffffffu, S3[i].y, off);
        S4[i].x += __shfl_xor_sync(0xffffffffu, S4[i].x, off); S4[i].y += __shfl_xor_sync(0xffffffffu, S4[i].y, off);
      }
    }
    if (seg == 0 && jr < n) {
      const int64_t idx = base + (l0 - m) + jr;
#pragma unroll
      for (int i = 0; i < NB; ++i) {
        if (b0 + i >= bofs + Bc) break;
        double2 G, C;
        if (!odd) {  // G = -S1 - i S2, C = i S3 - S4
          G = make_double2(-S1[i].x + S2[i].y, -S1[i].y - S2[i].x);
          C = make_double2(-S3[i].y - S4[i].x, S3[i].x - S4[i].y);
        } else {     // G = -S3 - i S4, C = i S1 - S2
          G = make_double2(-S3[i].x + S4[i].y, -S3[i].y - S4[i].x);
          C = make_double2(-S1[i].y - S2[i].x, S1[i].x - S2[i].y);
        }
        const int64_t o = ((int64_t(tile) * nalm + idx) * Bc + (b0 - bofs) + i) * 2;
        partial[o] = G;
        partial[o + 1] = C;
      }
    }
    __syncthreads();
  }
}

// =====================================================================
// layout kernels
// alm [B][ncomp][nalm] -> almT [nalm][B][ncomp]
__global__ void alm_to_T(const double2* __restrict__ alm, double2* __restrict__ almT, int B, int ncomp,
                         int64_t nalm) {
  const int64_t n = nalm * B * ncomp;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < n; t += int64_t(gridDim.x) * blockDim.x) {
    const int c = int(t % ncomp);
    const int b = int((t / ncomp) % B);
    const int64_t idx = t / (int64_t(ncomp) * B);
    almT[t] = alm[(int64_t(b) * ncomp + c) * nalm + idx];
  }
}

// sum_t partial[t][nalm][B][ncomp] * scale -> alm [B][ncomp][nalm]
__global__ void reduce_partials(const double2* __restrict__ partial, double2* __restrict__ alm, int ntiles, int B,
                                int ncomp, int64_t nalm, double scale, int bofs) {
  const int64_t n = nalm * B * ncomp;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < n; t += int64_t(gridDim.x) * blockDim.x) {
    double2 s = make_double2(0.0, 0.0);
    for (int i = 0; i < ntiles; ++i) s = cadd(s, partial[int64_t(i) * n + t]);
    const int c = int(t % ncomp);
    const int b = int((t / ncomp) % B);
    const int64_t idx = t / (int64_t(ncomp) * B);
    alm[(int64_t(bofs + b) * ncomp + c) * nalm + idx] = cscale(s, scale);
  }
}

// ---------------------------------------------------------------- launchers
// algorithmic Legendre work of one transform: 4 Rh nalm flops per spin-0 map,
// 16 Rh nalm per spin-s (G, C) pair; bytes: alm in + per-ring phases out
static double leg_flops(const Plan& P, int B, int spin) {
  return double(spin == 0 ? 4 : 16) * double(P.Rh) * double(P.nalm) * B;
}
static double leg_bytes(const Plan& P, int B, int spin) {
  const double nf = double(B) * (spin == 0 ? 1 : 2);
  return nf * 16.0 * (double(P.nalm) + double(P.R) * (P.mmax + 1));
}

int launch_legendre_synth_f64(const Plan& P, const double2* almT, double2* phase, int B, int spin,
                              cudaStream_t st) {
  StatScope sc(PS_K_LEG_SYNTH, leg_flops(P, B, spin), leg_bytes(P, B, spin), st);
  dim3 grid((P.Rh + SYN_THREADS - 1) / SYN_THREADS, P.mmax + 1, 1);
  const int t = P.tile[0][spin];
  if (spin == 0) {
    if (t ? t == 4 : B >= 4) {
      grid.z = (B + 3) / 4;
      synth0_f64<4><<<grid, SYN_THREADS, 0, st>>>(P.d_rings, P.d_mnorm0, almT, phase, P.R, P.Rh, P.lmax, P.mmax, B);
    } else {
      grid.z = B;
      synth0_f64<1><<<grid, SYN_THREADS, 0, st>>>(P.d_rings, P.d_mnorm0, almT, phase, P.R, P.Rh, P.lmax, P.mmax, B);
    }
  } else {
    if (!P.d_seed[spin]) return PS_ERR_INVALID;
    if (t ? t == 2 : B >= 2) {
      grid.z = (B + 1) / 2;
      synthS_f64<2><<<grid, SYN_THREADS, 0, st>>>(P.d_rings, P.d_seed[spin], almT, phase, P.R, P.Rh, P.lmax,
                                                  P.mmax, B, spin);
    } else {
      grid.z = B;
      synthS_f64<1><<<grid, SYN_THREADS, 0, st>>>(P.d_rings, P.d_seed[spin], almT, phase, P.R, P.Rh, P.lmax,
                                                  P.mmax, B, spin);
    }
  }
  PS_LAUNCH_CHECK();
  return PS_OK;
}

int adjoint_tiles(const Plan& P) { return (P.Rh + ADJ_THREADS - 1) / ADJ_THREADS; }

// maps [bofs, bofs + Bc) of a batch of B; partial holds [tile][nalm][Bc][ncomp]
int launch_legendre_adjoint_f64(const Plan& P, const double2* phase, double2* partial, int B, int bofs, int Bc,
                                int spin, cudaStream_t st) {
  StatScope sc(PS_K_LEG_ADJOINT, leg_flops(P, Bc, spin), leg_bytes(P, Bc, spin), st);
  dim3 grid(adjoint_tiles(P), P.mmax + 1, 1);
  const int t = P.tile[1][spin];
  if (spin == 0) {
    if (t ? t == 4 : Bc >= 4) {
      grid.z = (Bc + 3) / 4;
      adj0_f64<4><<<grid, ADJ_THREADS, 0, st>>>(P.d_rings, P.d_mnorm0, phase, partial, P.R, P.Rh, P.lmax, P.mmax,
                                                B, bofs, Bc, P.nalm);
    } else {
      grid.z = Bc;
      adj0_f64<1><<<grid, ADJ_THREADS, 0, st>>>(P.d_rings, P.d_mnorm0, phase, partial, P.R, P.Rh, P.lmax, P.mmax,
                                                B, bofs, Bc, P.nalm);
    }
  } else {
    if (!P.d_seed[spin]) return PS_ERR_INVALID;
    // one map per CTA: two maps would exceed the 48 KB of static shared memory
    grid.z = Bc;
    adjS_f64<1><<<grid, ADJ_THREADS, 0, st>>>(P.d_rings, P.d_seed[spin], phase, partial, P.R, P.Rh, P.lmax,
                                              P.mmax, B, bofs, Bc, P.nalm, spin);
  }
  PS_LAUNCH_CHECK();
  return PS_OK;
}

int launch_alm_to_T(const double2* alm, double2* almT, int B, int ncomp, int64_t nalm, int sms, cudaStream_t st) {
  const int64_t n = nalm * B * ncomp;
  int blocks = (int)std::min<int64_t>((n + 255) / 256, int64_t(sms) * 8);
  if (blocks < 1) blocks = 1;
  StatScope sc(PS_K_LAYOUT, 0.0, 32.0 * n, st);
  alm_to_T<<<blocks, 256, 0, st>>>(alm, almT, B, ncomp, nalm);
  PS_LAUNCH_CHECK();
  return PS_OK;
}

int launch_reduce_partials(const double2* partial, double2* alm, int ntiles, int B, int ncomp, int64_t nalm,
                           double scale, int bofs, int sms, cudaStream_t st) {
  const int64_t n = nalm * B * ncomp;
  int blocks = (int)std::min<int64_t>((n + 255) / 256, int64_t(sms) * 8);
  if (blocks < 1) blocks = 1;
  StatScope sc(PS_K_LAYOUT, 0.0, 16.0 * n * (ntiles + 1), st);
  reduce_partials<<<blocks, 256, 0, st>>>(partial, alm, ntiles, B, ncomp, nalm, scale, bofs);
  PS_LAUNCH_CHECK();
  return PS_OK;
}

}  // namespace ps
