// Mixed-precision Legendre stage of the adjoint (map -> alm direction).
//
// a_lm = sum_rings lam_lm(theta_r) P_m(r) (and the spin-s analogue, see the
// FP64 kernels for the parity and sign rules).  The recurrences run in FP64
// exactly as in the FP64 kernels; each CTA (a tile of 128 ring pairs, one order
// m, NB maps) drops the FP32-rounded values into a shared [32 l][128 ring] tile
// and reduces it against the FP32 per-ring phases of NB maps with FP32 FMAs
// (each thread two l of equal parity and a strided eighth of the rings, the
// eighths of a warp combined by shuffles).  The per-tile partial sums (FP32) are added in FP64,
// in a fixed order, by reduce_partials_f32.
#include <atomic>

#include "ps_common.cuh"
#include "ps_stats.cuh"

namespace ps {

constexpr int MX_THREADS = 128;  // ring pairs per CTA
constexpr int MX_LCH = 32;       // l per chunk (each reducing thread takes l offsets jr and jr + 16)

__device__ __forceinline__ void mx_seed0(int m, double sth, double mnorm, double& v, int& k) {
  Scaled s = smul(spow(sth, m), snorm(mnorm));
  to_kscale(s, v, k);
  if (m & 1) v = -v;
}

__device__ __forceinline__ void mx_seedS(int m, int s, const RingInfo& g, SeedNorm nrm, double& f, double& gg,
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

__device__ __forceinline__ float2 ffma2(float s, float2 a, float2 acc) {
  return make_float2(fmaf(s, a.x, acc.x), fmaf(s, a.y, acc.y));
}

// reduction mapping of the 4 warps: warp w -> parity p = w & 1, jset = w >> 1;
// lane -> jq = lane >> 3, seg = lane & 7; l offsets jr = p + 2 (4 jset + jq)
// and jr + 16 (same parity, sharing the phase loads); rings seg, seg + 8, ..., seg + 120

// spin 0.  phase [R][mmax+1][B] (complex64) -> partial [tile][nalm][B] (complex64)
template <int NB>
__global__ void __launch_bounds__(MX_THREADS) adj0_mx(const RingInfo* __restrict__ rings,
                                                       const double* __restrict__ mnorm,
                                                       const float2* __restrict__ phase,
                                                       float2* __restrict__ partial, int R, int Rh, int lmax,
                                                       int mmax, int B, int bofs, int Bc, int64_t nalm) {
  const int m = blockIdx.y, tile = blockIdx.x, tid = threadIdx.x;
  const int rp = tile * MX_THREADS + tid;
  const int b0 = bofs + blockIdx.z * NB;
  // ring-contiguous layouts: a warp's 8 ring segments read 8 consecutive
  // words (no bank conflicts); the l rows are padded by 4 words
  __shared__ float s_lam[MX_LCH][MX_THREADS + 4];
  __shared__ float2 s_P[2][NB][MX_THREADS];  // [N+S, N-S][map][ring]
  __shared__ double s_a[MX_LCH], s_b[MX_LCH];
  const bool active = rp < Rh;
  const RingInfo g = rings[active ? rp : 0];
  const int rs = R - 1 - rp;
#pragma unroll
  for (int i = 0; i < NB; ++i) {
    float2 pn = make_float2(0.f, 0.f), ps_ = pn;
    if (active && b0 + i < bofs + Bc) {
      pn = phase[(int64_t(rp) * (mmax + 1) + m) * B + b0 + i];
      if (rs != rp) ps_ = phase[(int64_t(rs) * (mmax + 1) + m) * B + b0 + i];
    }
    s_P[0][i][tid] = make_float2(pn.x + ps_.x, pn.y + ps_.y);
    s_P[1][i][tid] = make_float2(pn.x - ps_.x, pn.y - ps_.y);
  }
  const double x = g.z;
  double cur, prev = 0.0;
  int k;
  mx_seed0(m, g.sth, mnorm[m], cur, k);
  if (!active) { cur = 0.0; k = 0; }
  const int warp = tid >> 5, lane = tid & 31;
  const int p = warp & 1, jset = warp >> 1, jq = lane >> 3, seg = lane & 7;
  const int jr = p + 2 * (4 * jset + jq);
  const int64_t base = alm_index(m, m, lmax);
  for (int l0 = m; l0 <= lmax; l0 += MX_LCH) {
    const int n = min(MX_LCH, lmax - l0 + 1);
    if (tid < MX_LCH) {
      double a = 0.0, b = 0.0;
      const int l = l0 + tid + 1;
      if (l <= lmax) {
        const double mm = double(m) * m;
        a = sqrt((4.0 * l * l - 1.0) / (double(l) * l - mm));
        if (l >= m + 2) b = a / sqrt((4.0 * (l - 1.0) * (l - 1.0) - 1.0) / ((l - 1.0) * (l - 1.0) - mm));
      }
      s_a[tid] = a;
      s_b[tid] = b;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < MX_LCH; ++j) {
      s_lam[j][tid] = (k == 0) ? float(cur) : 0.f;
      const double nxt = s_a[j] * x * cur - s_b[j] * prev;
      prev = cur;
      cur = nxt;
      if (k < 0 && fabs(cur) > PS_FTHRESH) { cur *= PS_FSMALL; prev *= PS_FSMALL; ++k; }
    }
    __syncthreads();
    float2 acc[2][NB];
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
      for (int i = 0; i < NB; ++i) acc[h][i] = make_float2(0.f, 0.f);
#pragma unroll 2
    for (int t = 0; t < MX_THREADS / 8; ++t) {
      const int r = seg + 8 * t;
      const float lam0 = s_lam[jr][r], lam1 = s_lam[jr + 16][r];
#pragma unroll
      for (int i = 0; i < NB; ++i) {
        const float2 pv = s_P[p][i][r];
        acc[0][i] = ffma2(lam0, pv, acc[0][i]);
        acc[1][i] = ffma2(lam1, pv, acc[1][i]);
      }
    }
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
      for (int i = 0; i < NB; ++i) {
#pragma unroll
        for (int off = 1; off < 8; off <<= 1) {
          acc[h][i].x += __shfl_xor_sync(0xffffffffu, acc[h][i].x, off);
          acc[h][i].y += __shfl_xor_sync(0xffffffffu, acc[h][i].y, off);
        }
      }
    if (seg == 0) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int jj = jr + 16 * h;
        if (jj >= n) continue;
        const int64_t idx = base + (l0 - m) + jj;
#pragma unroll
        for (int i = 0; i < NB; ++i)
          if (b0 + i < bofs + Bc) partial[(int64_t(tile) * nalm + idx) * Bc + (b0 - bofs) + i] = acc[h][i];
      }
    }
    __syncthreads();
  }
}

// dynamic shared memory of adjS_mx (above the 48 KB static limit for NB = 4)
template <int NB>
struct AdjSSmem {
  float fp[MX_LCH][MX_THREADS + 4];  // F+ of the chunk, ring-contiguous rows (padded against bank conflicts)
  float fm[MX_LCH][MX_THREADS + 4];  // F-
  float2 Q[2][NB][MX_THREADS];       // [N+S, N-S][map][ring]
  float2 U[2][NB][MX_THREADS];
  double A[MX_LCH], D[MX_LCH], C[MX_LCH];
};

// spin s.  phase [R][mmax+1][B][2] (Q, U) -> partial [tile][nalm][B][2] (G, C)
template <int NB>
__global__ void __launch_bounds__(MX_THREADS) adjS_mx(const RingInfo* __restrict__ rings,
                                                       const SeedNorm* __restrict__ seednorm,
                                                       const float2* __restrict__ phase,
                                                       float2* __restrict__ partial, int R, int Rh, int lmax,
                                                       int mmax, int B, int bofs, int Bc, int64_t nalm, int spin) {
  const int m = blockIdx.y, tile = blockIdx.x, tid = threadIdx.x;
  const int rp = tile * MX_THREADS + tid;
  const int b0 = bofs + blockIdx.z * NB;
  extern __shared__ __align__(16) unsigned char mx_smem[];
  AdjSSmem<NB>& sm = *reinterpret_cast<AdjSSmem<NB>*>(mx_smem);
  auto& s_fp = sm.fp;
  auto& s_fm = sm.fm;
  auto& s_Q = sm.Q;
  auto& s_U = sm.U;
  auto& s_A = sm.A;
  auto& s_D = sm.D;
  auto& s_C = sm.C;
  const bool active = rp < Rh;
  const RingInfo g = rings[active ? rp : 0];
  const int rs = R - 1 - rp;
#pragma unroll
  for (int i = 0; i < NB; ++i) {
    float2 qn = make_float2(0.f, 0.f), qs = qn, un = qn, us = qn;
    if (active && b0 + i < bofs + Bc) {
      const int64_t o = ((int64_t(rp) * (mmax + 1) + m) * B + b0 + i) * 2;
      qn = phase[o];
      un = phase[o + 1];
      if (rs != rp) {
        const int64_t o2 = ((int64_t(rs) * (mmax + 1) + m) * B + b0 + i) * 2;
        qs = phase[o2];
        us = phase[o2 + 1];
      }
    }
    s_Q[0][i][tid] = make_float2(qn.x + qs.x, qn.y + qs.y);
    s_Q[1][i][tid] = make_float2(qn.x - qs.x, qn.y - qs.y);
    s_U[0][i][tid] = make_float2(un.x + us.x, un.y + us.y);
    s_U[1][i][tid] = make_float2(un.x - us.x, un.y - us.y);
  }
  const double x = g.z;
  const int lmin = max(m, spin);
  double sf, sg;
  int k;
  mx_seedS(m, spin, g, seednorm[m], sf, sg, k);
  if (!active) { sf = 0.0; sg = 0.0; k = 0; }
  double f = 0.0, gg = 0.0, fpv = 0.0, gpv = 0.0;
  const int warp = tid >> 5, lane = tid & 31;
  const int p = warp & 1, jset = warp >> 1, jq = lane >> 3, seg = lane & 7;
  const int jr = p + 2 * (4 * jset + jq);
  // F+ multiplies (N + (-1)^p S), F- multiplies (N - (-1)^p S)
  const int cplus = p, cminus = 1 - p;
  const bool odd = spin & 1;
  const int64_t base = alm_index(m, m, lmax);
  for (int l0 = m; l0 <= lmax; l0 += MX_LCH) {
    const int n = min(MX_LCH, lmax - l0 + 1);
    if (tid < MX_LCH) {
      double A = 0.0, D = 0.0, C = 0.0;
      const int l = l0 + tid;
      if (l >= lmin && l < lmax) {
        auto rho = [&](double L) {
          return sqrt(fmax(L * L - double(m) * m, 0.0) * fmax(L * L - double(spin) * spin, 0.0));
        };
        const double r1 = rho(l + 1.0), q = sqrt((2.0 * l + 3.0) * (2.0 * l + 1.0));
        A = q * (l + 1.0) / r1;
        D = q * double(m) * double(spin) / (double(l) * r1);
        C = sqrt((2.0 * l + 3.0) / (2.0 * l - 1.0)) * (l + 1.0) * rho(double(l)) / (double(l) * r1);
      }
      s_A[tid] = A; s_D[tid] = D; s_C[tid] = C;
    }
    __syncthreads();
#pragma unroll 4
    for (int j = 0; j < MX_LCH; ++j) {
      if (l0 + j == lmin) { f = sf; gg = sg; fpv = 0.0; gpv = 0.0; }
      s_fp[j][tid] = (k == 0) ? float(0.5 * (f + gg)) : 0.f;
      s_fm[j][tid] = (k == 0) ? float(0.5 * (f - gg)) : 0.f;
      const double ax = s_A[j] * x;
      const double fn = (ax + s_D[j]) * f - s_C[j] * fpv;
      const double gn = (ax - s_D[j]) * gg - s_C[j] * gpv;
      fpv = f; f = fn; gpv = gg; gg = gn;
      if (k < 0 && fmax(fabs(f), fabs(gg)) > PS_FTHRESH) {
        f *= PS_FSMALL; fpv *= PS_FSMALL; gg *= PS_FSMALL; gpv *= PS_FSMALL; ++k;
      }
    }
    __syncthreads();
    float2 S1[2][NB], S2[2][NB], S3[2][NB], S4[2][NB];
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
      for (int i = 0; i < NB; ++i) {
        S1[h][i] = make_float2(0.f, 0.f); S2[h][i] = S1[h][i]; S3[h][i] = S1[h][i]; S4[h][i] = S1[h][i];
      }
#pragma unroll 2
    for (int t = 0; t < MX_THREADS / 8; ++t) {
      const int r = seg + 8 * t;
      const float vp0 = s_fp[jr][r], vm0 = s_fm[jr][r], vp1 = s_fp[jr + 16][r], vm1 = s_fm[jr + 16][r];
#pragma unroll
      for (int i = 0; i < NB; ++i) {
        const float2 qp = s_Q[cplus][i][r], qm = s_Q[cminus][i][r], up = s_U[cplus][i][r], um = s_U[cminus][i][r];
        S1[0][i] = ffma2(vp0, qp, S1[0][i]); S1[1][i] = ffma2(vp1, qp, S1[1][i]);
        S2[0][i] = ffma2(vm0, um, S2[0][i]); S2[1][i] = ffma2(vm1, um, S2[1][i]);
        S3[0][i] = ffma2(vm0, qm, S3[0][i]); S3[1][i] = ffma2(vm1, qm, S3[1][i]);
        S4[0][i] = ffma2(vp0, up, S4[0][i]); S4[1][i] = ffma2(vp1, up, S4[1][i]);
      }
    }
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
      for (int i = 0; i < NB; ++i) {
#pragma unroll
        for (int off = 1; off < 8; off <<= 1) {
          S1[h][i].x += __shfl_xor_sync(0xffffffffu, S1[h][i].x, off); S1[h][i].y += __shfl_xor_sync(0xffffffffu, S1[h][i].y, off);
          S2[h][i].x += __shfl_xor_sync(0xffffffffu, S2[h][i].x, off); S2[h][i].y += __shfl_xor_sync(0xffffffffu, S2[h][i].y, off);
          S3[h][i].x += __shfl_xor_sync(0xffffffffu, S3[h][i].x, off); S3[h][i].y += __shfl_xor_sync(0xffffffffu, S3[h][i].y, off);
          S4[h][i].x += __shfl_xor_sync(0xffffffffu, S4[h][i].x, off); S4[h][i].y += __shfl_xor_sync(0xffffffffu, S4[h][i].y, off);
        }
      }
    if (seg == 0) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int jj = jr + 16 * h;
        if (jj >= n) continue;
        const int64_t idx = base + (l0 - m) + jj;
#pragma unroll
        for (int i = 0; i < NB; ++i) {
          if (b0 + i >= bofs + Bc) break;
          float2 G, C;
          if (!odd) {  // G = -S1 - i S2, C = i S3 - S4
            G = make_float2(-S1[h][i].x + S2[h][i].y, -S1[h][i].y - S2[h][i].x);
            C = make_float2(-S3[h][i].y - S4[h][i].x, S3[h][i].x - S4[h][i].y);
          } else {     // G = -S3 - i S4, C = i S1 - S2
            G = make_float2(-S3[h][i].x + S4[h][i].y, -S3[h][i].y - S4[h][i].x);
            C = make_float2(-S1[h][i].y - S2[h][i].x, S1[h][i].x - S2[h][i].y);
          }
          const int64_t o = ((int64_t(tile) * nalm + idx) * Bc + (b0 - bofs) + i) * 2;
          partial[o] = G;
          partial[o + 1] = C;
        }
      }
    }
    __syncthreads();
  }
}

// sum_t partial[t][nalm][B][ncomp] (FP32) in FP64, times scale -> alm [B][ncomp][nalm] (FP64)
__global__ void reduce_partials_f32(const float2* __restrict__ partial, double2* __restrict__ alm, int ntiles,
                                    int B, int ncomp, int64_t nalm, double scale, int bofs) {
  const int64_t n = nalm * B * ncomp;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < n; t += int64_t(gridDim.x) * blockDim.x) {
    double sx = 0.0, sy = 0.0;
    for (int i = 0; i < ntiles; ++i) {
      const float2 v = partial[int64_t(i) * n + t];
      sx += double(v.x);
      sy += double(v.y);
    }
    const int c = int(t % ncomp);
    const int b = int((t / ncomp) % B);
    const int64_t idx = t / (int64_t(ncomp) * B);
    alm[(int64_t(bofs + b) * ncomp + c) * nalm + idx] = make_double2(sx * scale, sy * scale);
  }
}

int mx_adjoint_tiles(const Plan& P) { return (P.Rh + MX_THREADS - 1) / MX_THREADS; }

// maps [bofs, bofs + Bc) of a batch of B; partial holds [tile][nalm][Bc][ncomp]
int launch_legendre_adjoint_mx(const Plan& P, const float2* phase, float2* partial, int B, int bofs, int Bc,
                               int spin, cudaStream_t st) {
  const double flops = double(spin == 0 ? 4 : 16) * double(P.Rh) * double(P.nalm) * Bc;
  const double bytes = double(Bc) * (spin == 0 ? 1 : 2) * (8.0 * P.R * (P.mmax + 1) + 8.0 * P.nalm * mx_adjoint_tiles(P));
  StatScope sc(PS_K_LEG_ADJOINT, flops, bytes, st);
  dim3 grid(mx_adjoint_tiles(P), P.mmax + 1, 1);
  const int t = P.tile[1][spin];
  if (spin == 0) {
    if (t ? t == 8 : Bc >= 8) {
      grid.z = (Bc + 7) / 8;
      adj0_mx<8><<<grid, MX_THREADS, 0, st>>>(P.d_rings, P.d_mnorm0, phase, partial, P.R, P.Rh, P.lmax, P.mmax, B,
                                              bofs, Bc, P.nalm);
    } else {
      grid.z = Bc;
      adj0_mx<1><<<grid, MX_THREADS, 0, st>>>(P.d_rings, P.d_mnorm0, phase, partial, P.R, P.Rh, P.lmax, P.mmax, B,
                                              bofs, Bc, P.nalm);
    }
  } else {
    if (!P.d_seed[spin]) return PS_ERR_INVALID;
    if (t ? t == 4 : Bc >= 4) {
      grid.z = (Bc + 3) / 4;
      const int smem = int(sizeof(AdjSSmem<4>));
      // the opt-in attribute is per device: remember the devices it was set on
      static std::atomic<uint64_t> attr_set{0};
      int dev = 0;
      if (cudaGetDevice(&dev) != cudaSuccess) return PS_ERR_CUDA;
      const uint64_t bit = uint64_t(1) << (dev & 63);
      if (!(attr_set.load() & bit)) {
        if (cudaFuncSetAttribute(adjS_mx<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
          return PS_ERR_CUDA;
        attr_set.fetch_or(bit);
      }
      adjS_mx<4><<<grid, MX_THREADS, smem, st>>>(P.d_rings, P.d_seed[spin], phase, partial, P.R, P.Rh, P.lmax, P.mmax,
                                              B, bofs, Bc, P.nalm, spin);
    } else {
      grid.z = Bc;
      adjS_mx<1><<<grid, MX_THREADS, sizeof(AdjSSmem<1>), st>>>(P.d_rings, P.d_seed[spin], phase, partial, P.R, P.Rh, P.lmax, P.mmax,
                                              B, bofs, Bc, P.nalm, spin);
    }
  }
  PS_LAUNCH_CHECK();
  return PS_OK;
}

int launch_reduce_partials_f32(const float2* partial, double2* alm, int ntiles, int B, int ncomp, int64_t nalm,
                               double scale, int bofs, int sms, cudaStream_t st) {
  const int64_t n = nalm * B * ncomp;
  int blocks = (int)std::min<int64_t>((n + 255) / 256, int64_t(sms) * 8);
  if (blocks < 1) blocks = 1;
  StatScope sc(PS_K_LAYOUT, 0.0, 8.0 * n * ntiles + 16.0 * n, st);
  reduce_partials_f32<<<blocks, 256, 0, st>>>(partial, alm, ntiles, B, ncomp, nalm, scale, bofs);
  PS_LAUNCH_CHECK();
  return PS_OK;
}

}  // namespace ps
