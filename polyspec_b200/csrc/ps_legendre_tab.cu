// Table-driven mixed-precision Legendre stages on the tensor cores (tcgen05,
// kind::tf32, accumulators in TMEM).
//
// The normalised Legendre values of a plan do not depend on the data, so for
// a mixed-precision plan they can be computed once (FP64 recurrence with the
// scaled seeds of the on-the-fly kernels, rounded to FP32) and kept in HBM in
// the order in which the two GEMMs below consume them.  Each transform then
// streams the table instead of re-running the recurrence for every group of
// maps: at Nside 1024, lmax 2048 the spin-0 table is 17.7 GB and the spin-s
// table (F+ and F-) 35.4 GB, read once per map group of a transform (up to
// 64 maps of spin 0, 16 (synthesis) or 32 (adjoint) of spin s).
//
// Table layout.  For each order m the l range [m, lmax] is cut into blocks of
// 64 consecutive l; inside a block the 64 positions are sorted by parity of
// l - m: position j < 32 holds l = m + 64b + 2j, position 32 + j holds
// l = m + 64b + 2j + 1 (zero beyond lmax).  Ring pairs (north ring and its
// mirror, the equator last) are grouped in quads of 4; one unit
// (m, block b, quad q) is [ncomp][64 positions][4 rings] FP32 (ncomp 1 for
// spin 0, 2 for spin s: F+ then F-), and units are stored in the order
// (m, b, q).  A float4 of a unit is four consecutive rings at one l, which is
// one 16-byte row of a K-major core matrix of the adjoint's A operand (K =
// rings); the synthesis (K = l) transposes 4 x 4 blocks in registers.
//
// Both GEMMs split every FP32 operand into TF32 hi + lo and issue three MMAs
// per K step (hi.hi + hi.lo + lo.hi).  The tensor core's FP32 accumulation
// truncates, so the accumulator D is restarted for every stage of 32 K values
// and added into a running sum S that also lives in TMEM (round-to-nearest
// FP32 adds by the drain warps).  TMEM: D[2 accumulators][128 columns] and
// S[2][128], all 512 columns of the SM: one CTA of 16 warps per SM, the four
// warps that share a TMEM lane quarter splitting the columns between them.
//
// Columns of D are (part, map) with the part index outermost: spin 0
// (re, im) of the complex value, spin s four real parts; map group g of up
// to 64 (spin 0) or 16 / 32 (spin s synthesis / adjoint) maps.  N = the used
// columns rounded up to 16.
//
// Staging.  The table tiles of the next two stages (and, in the spin-s
// adjoint, the phase rows of the stage's rings) are fetched by bulk copies
// (cp.async.bulk with mbarrier transaction counts) into two shared buffers
// while the current stage is split and multiplied; the a_lm (synthesis) and
// spin-0 phases (adjoint) of the next stage are loaded into registers.
//
// Synthesis (alm -> ring phases), CTA = (map group, ring tile of 128 ring
// pairs, m): M = ring pairs, K = l, two accumulators.  Spin 0: accumulator p
// sums the l of parity p; north ring = S0 + S1, south = S0 - S1.  Spin s:
// W = sum_even F+ u + sum_odd F- v and V = sum_odd F+ u + sum_even F- v (u, v
// the (Q, U) contributions of (G, C) through F+ and F-); north = W + V,
// south = W - V.  The A row of ring 4q + i of the tile is 32 i + q, so that
// the 16-byte stores of eight consecutive lanes (consecutive q) fall into
// eight different bank groups.
//
// Adjoint (ring phases -> alm), CTA = (map group, group of 4 l blocks, m):
// M = 128 l of one parity (32 positions of each of the 4 blocks), K = rings
// (32 per stage for spin 0; for spin s 16 rings as F+ rows and the same 16 as
// F- rows), two accumulators (parity 0 and 1) against the ring sums N + S
// and differences N - S.  The output is written straight into the caller's
// alm (FP64, times scale and an optional per-lm factor): there are no
// per-ring-tile partial sums.
//
// Every mbarrier wait is bounded; on expiry the kernel raises the plan's
// error flag, waits once more (bounded) for the MMAs it issued and frees its
// TMEM.
#include <algorithm>
#include <vector>

#include "ps_common.cuh"
#include "ps_stats.cuh"
#include "ps_tc.cuh"

namespace ps {

constexpr int TB_LB = 64;        // l per table block
constexpr int TB_TILE = 128;     // ring pairs per synthesis tile (MMA M)
constexpr int TB_THREADS = 128;  // table generation
constexpr int TM_THREADS = 512;  // the two GEMMs: 16 warps, 4 per TMEM lane quarter
constexpr uint32_t TB_WAIT_LIMIT = 1u << 24;

// ------------------------------------------------------------------ table geometry
// number of table blocks of order m
__host__ __device__ __forceinline__ int tab_nblocks(int m, int lmax) { return (lmax - m) / TB_LB + 1; }
// l of position pos of block b (may exceed lmax)
__host__ __device__ __forceinline__ int tab_l(int m, int b, int pos) {
  return m + TB_LB * b + 2 * (pos & 31) + (pos >> 5);
}

// ------------------------------------------------------------------ recurrence (as the FP64 kernels)
__device__ __forceinline__ void tab_seed0(int m, double sth, double mnorm, double& v, int& k) {
  Scaled s = smul(spow(sth, m), snorm(mnorm));
  to_kscale(s, v, k);
  if (m & 1) v = -v;
}

__device__ __forceinline__ void tab_seedS(int m, int s, const RingInfo& g, SeedNorm nrm, double& f, double& gg,
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

// One CTA = 128 ring pairs of one order m; thread = ring pair.  Block by block the
// values go to a padded shared stage [32 quads][unit + 4 floats] and then out to
// the table as 32 contiguous units.
template <int NOPS>
__global__ void __launch_bounds__(TB_THREADS) tab_gen_kernel(const RingInfo* __restrict__ rings,
                                                             const double* __restrict__ mnorm,
                                                             const SeedNorm* __restrict__ seednorm, int Rh, int lmax,
                                                             int spin, const int64_t* __restrict__ blockoff,
                                                             int nquads, float* __restrict__ table) {
  constexpr int UNIT = NOPS * TB_LB * 4;  // floats per unit
  constexpr int USTR = UNIT + 4;          // padded stride in the stage
  extern __shared__ __align__(16) float tg_stage[];  // [32][USTR]
  __shared__ double s_c0[TB_LB], s_c1[TB_LB], s_c2[TB_LB];
  const int m = blockIdx.y, tile = blockIdx.x, tid = threadIdx.x;
  const int rp = tile * TB_TILE + tid;
  const bool active = rp < Rh;
  const RingInfo g = rings[active ? rp : 0];
  const double x = g.z;
  const int lmin = NOPS == 1 ? m : max(m, spin);
  double f = 0.0, fp = 0.0, gg = 0.0, gp = 0.0, sf = 0.0, sg = 0.0;
  int k = 0;
  if (NOPS == 1) tab_seed0(m, g.sth, mnorm[m], f, k);
  else tab_seedS(m, spin, g, seednorm[m], sf, sg, k);
  if (!active) { f = 0.0; sf = 0.0; sg = 0.0; k = 0; }
  float* my = tg_stage + (tid >> 2) * USTR + (tid & 3);
  const int nb = tab_nblocks(m, lmax);
  for (int b = 0; b < nb; ++b) {
    const int l0 = m + TB_LB * b;
    if (tid < TB_LB) {
      double c0 = 0.0, c1 = 0.0, c2 = 0.0;
      if (NOPS == 1) {  // lam_{l+1} = c0 x lam_l - c1 lam_{l-1}, l = l0 + tid
        const int l = l0 + tid + 1;
        if (l <= lmax) {
          const double mm = double(m) * m;
          c0 = sqrt((4.0 * l * l - 1.0) / (double(l) * l - mm));
          if (l >= m + 2) c1 = c0 / sqrt((4.0 * (l - 1.0) * (l - 1.0) - 1.0) / ((l - 1.0) * (l - 1.0) - mm));
        }
      } else {  // f_{l+1} = (c0 x + c1) f_l - c2 f_{l-1} (g with -c1)
        const int l = l0 + tid;
        if (l >= lmin && l < lmax) {
          auto rho = [&](double L) {
            return sqrt(fmax(L * L - double(m) * m, 0.0) * fmax(L * L - double(spin) * spin, 0.0));
          };
          const double r1 = rho(l + 1.0), q = sqrt((2.0 * l + 3.0) * (2.0 * l + 1.0));
          c0 = q * (l + 1.0) / r1;
          c1 = q * double(m) * double(spin) / (double(l) * r1);
          c2 = sqrt((2.0 * l + 3.0) / (2.0 * l - 1.0)) * (l + 1.0) * rho(double(l)) / (double(l) * r1);
        }
      }
      s_c0[tid] = c0; s_c1[tid] = c1; s_c2[tid] = c2;
    }
    __syncthreads();
    for (int j = 0; j < TB_LB; ++j) {
      const int l = l0 + j;
      const int pos = ((j & 1) << 5) | (j >> 1);
      if (NOPS == 1) {
        my[pos * 4] = (k == 0 && l <= lmax) ? float(f) : 0.f;
        const double nxt = s_c0[j] * x * f - s_c1[j] * fp;
        fp = f;
        f = nxt;
        if (k < 0 && fabs(f) > PS_FTHRESH) { f *= PS_FSMALL; fp *= PS_FSMALL; ++k; }
      } else {
        if (l == lmin) { f = sf; gg = sg; fp = 0.0; gp = 0.0; }
        const bool use = (k == 0) && (l <= lmax);
        my[pos * 4] = use ? float(0.5 * (f + gg)) : 0.f;
        my[(TB_LB + pos) * 4] = use ? float(0.5 * (f - gg)) : 0.f;
        const double ax = s_c0[j] * x;
        const double fn = (ax + s_c1[j]) * f - s_c2[j] * fp;
        const double gn = (ax - s_c1[j]) * gg - s_c2[j] * gp;
        fp = f; f = fn; gp = gg; gg = gn;
        if (k < 0 && fmax(fabs(f), fabs(gg)) > PS_FTHRESH) {
          f *= PS_FSMALL; fp *= PS_FSMALL; gg *= PS_FSMALL; gp *= PS_FSMALL; ++k;
        }
      }
    }
    __syncthreads();
    // 32 units of this tile are contiguous in the table
    float4* dst = reinterpret_cast<float4*>(table + ((blockoff[m] + b) * int64_t(nquads) + int64_t(tile) * 32) * UNIT);
    for (int i = tid; i < 32 * UNIT / 4; i += TB_THREADS) {
      const int q = i / (UNIT / 4), w = i % (UNIT / 4);
      dst[i] = *reinterpret_cast<const float4*>(tg_stage + q * USTR + 4 * w);
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------------ MMA helpers
__device__ __forceinline__ uint32_t kcore_off(int row, int kc) {
  return uint32_t(((row >> 3) * 2 + kc) * 128 + (row & 7) * 16);
}
__device__ __forceinline__ uint64_t kdesc(uint32_t saddr) {
  uint64_t d = 0;
  d |= uint64_t((saddr >> 4) & 0x3FFFu);
  d |= uint64_t(128u >> 4) << 16;  // leading (K) byte offset: the second 16-byte core matrix of a K step
  d |= uint64_t(256u >> 4) << 32;  // stride byte offset: the next 8-row group
  d |= uint64_t(1) << 46;          // descriptor version (sm_100)
  return d;                        // no swizzle
}
__device__ __forceinline__ void split4(float4 v, float4& hi, float4& lo) {
  hi.x = tc::tf32_rna(v.x); lo.x = tc::tf32_rna(v.x - hi.x);
  hi.y = tc::tf32_rna(v.y); lo.y = tc::tf32_rna(v.y - hi.y);
  hi.z = tc::tf32_rna(v.z); lo.z = tc::tf32_rna(v.z - hi.z);
  hi.w = tc::tf32_rna(v.w); lo.w = tc::tf32_rna(v.w - hi.w);
}
__device__ __forceinline__ void st_split(uint8_t* smem, uint32_t hi_off, uint32_t lo_off, float4 v) {
  float4 h, l;
  split4(v, h, l);
  *reinterpret_cast<float4*>(smem + hi_off) = h;
  *reinterpret_cast<float4*>(smem + lo_off) = l;
}
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const float* v) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], "
      "{%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(taddr),
      "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])), "r"(__float_as_uint(v[3])),
      "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])), "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])),
      "r"(__float_as_uint(v[8])), "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])), "r"(__float_as_uint(v[11])),
      "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])), "r"(__float_as_uint(v[14])),
      "r"(__float_as_uint(v[15]))
      : "memory");
}
__device__ __forceinline__ void tmem_st_wait() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// Shared-memory plan of both GEMMs (offsets from a 1024-byte aligned base):
//   A[acc][kstep][hi/lo]   4 KB each (128 rows x 8 K)          64 KB
//   B[acc][kstep][hi/lo]   NMAX x 32 B each                    16 NMAX x 32 B
//   STG[2]                 raw table tiles of the next stages, filled by bulk copies
//   MISC                   mbarriers (MMA done, staging buffer full x 2), TMEM slot
template <int NMAX, uint32_t STG_BYTES>
struct TabSmem {
  static constexpr int KS = 4;  // K steps (of 8) per accumulator and stage
  static constexpr uint32_t A_TILE = TB_TILE * 32;
  static constexpr uint32_t B_TILE = NMAX * 32;
  static constexpr uint32_t B_OFF = 2 * KS * 2 * A_TILE;
  static constexpr uint32_t STG_OFF = B_OFF + 2 * KS * 2 * B_TILE;
  static constexpr uint32_t MISC_OFF = STG_OFF + 2 * STG_BYTES;
  static constexpr uint32_t DYN = MISC_OFF + 64 + 1024;
  static constexpr uint32_t TMEM_COLS = 4 * NMAX;  // D[2][NMAX], S[2][NMAX]
  __device__ static uint32_t a(int acc, int ks, int hl) { return ((acc * KS + ks) * 2 + hl) * A_TILE; }
  __device__ static uint32_t b(int acc, int ks, int hl) { return B_OFF + ((acc * KS + ks) * 2 + hl) * B_TILE; }
  __device__ static uint32_t stg(int buf) { return STG_OFF + uint32_t(buf) * STG_BYTES; }
};

// CTA state shared by both GEMMs
struct TabCta {
  uint8_t* smem;
  uint32_t sbase;
  uint32_t mbar_mma;   // MMAs of the current stage complete
  uint32_t mbar_full;  // + 8 * buf: staging buffer buf filled
  uint32_t tmem;
};

template <class S>
__device__ __forceinline__ TabCta tab_begin(uint8_t* smem_raw) {
  TabCta c;
  c.smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  c.sbase = tc::smem_u32(c.smem);
  c.mbar_mma = c.sbase + S::MISC_OFF;
  c.mbar_full = c.sbase + S::MISC_OFF + 8;
  uint32_t* slot = reinterpret_cast<uint32_t*>(c.smem + S::MISC_OFF + 32);
  if ((threadIdx.x >> 5) == 0) {
    tc::tmem_alloc(tc::smem_u32(slot), S::TMEM_COLS);
    tc::tmem_relinquish();
  }
  if (threadIdx.x == 0) {
    tc::mbar_init(c.mbar_mma, 1);
    tc::mbar_init(c.mbar_full, 1);
    tc::mbar_init(c.mbar_full + 8, 1);
    tc::fence_mbar_init();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  c.tmem = *slot;
  return c;
}

// one stage's MMAs: 2 accumulators x 4 K steps x (hi.hi + hi.lo + lo.hi), D fresh per stage
template <class S, int NMAX>
__device__ __forceinline__ void tab_issue(uint32_t sbase, uint32_t tmem, uint32_t idesc) {
#pragma unroll
  for (int acc = 0; acc < 2; ++acc) {
    const uint32_t d = tmem + uint32_t(acc * NMAX);
#pragma unroll
    for (int ks = 0; ks < S::KS; ++ks) {
      const uint64_t ah = kdesc(sbase + S::a(acc, ks, 0)), al = kdesc(sbase + S::a(acc, ks, 1));
      const uint64_t bh = kdesc(sbase + S::b(acc, ks, 0)), bl = kdesc(sbase + S::b(acc, ks, 1));
      tc::mma_tf32(d, ah, bh, idesc, ks > 0 ? 1u : 0u);
      tc::mma_tf32(d, ah, bl, idesc, 1u);
      tc::mma_tf32(d, al, bh, idesc, 1u);
    }
  }
}

// S += D for this thread's TMEM lane (first stage: S = D), columns [0, n) of both accumulators.
// Unit u = (16-column chunk u >> 1, accumulator u & 1); the TM_THREADS / 128 warps that share a TMEM
// lane quarter take every fourth unit; the loads of D and S of a unit share one wait
template <int NMAX>
__device__ __forceinline__ void tab_drain(uint32_t lane_addr, int n, bool first) {
  const int nu = n >> 3;
#pragma unroll 1
  for (int u = int(threadIdx.x >> 7); u < nu; u += TM_THREADS / 128) {
    float d[16], s[16];
    const uint32_t dc = lane_addr + uint32_t((u & 1) * NMAX + 16 * (u >> 1));
    const uint32_t sc = dc + uint32_t(2 * NMAX);
    tc::tmem_ld16(dc, d);
    if (!first) tc::tmem_ld16(sc, s);
    tc::tmem_ld_wait();
    if (!first) {
#pragma unroll
      for (int q = 0; q < 16; ++q) d[q] += s[q];
    }
    tmem_st16(sc, d);
  }
  tmem_st_wait();
}

// bounded wait of every thread on an mbarrier phase; on expiry raise the flag
__device__ __forceinline__ bool tab_wait(uint32_t mbar, uint32_t parity, int* err_flag) {
  const bool ok = __syncthreads_and(tc::mbar_wait_bounded(mbar, parity, TB_WAIT_LIMIT));
  if (!ok && threadIdx.x == 0) atomicExch(err_flag, 1);
  return ok;
}

// make every thread's operand stores visible to the tensor core, then (thread 0) issue the MMAs
template <class S, int NMAX>
__device__ __forceinline__ void tab_issue_stage(const TabCta& c, uint32_t idesc) {
  tc::fence_proxy_async();
  __syncthreads();
  if (threadIdx.x == 0) {
    tc::fence_after_sync();
    tab_issue<S, NMAX>(c.sbase, c.tmem, idesc);
    tc::mma_commit(c.mbar_mma);
  }
}

// wait for the stage's MMAs and drain D into S; false (flag raised) when the wait expires
template <int NMAX>
__device__ __forceinline__ bool tab_finish_stage(const TabCta& c, int n, bool first, uint32_t& phase,
                                                 int* err_flag) {
  if (!tab_wait(c.mbar_mma, phase, err_flag)) {
    tc::mbar_wait_bounded(c.mbar_mma, phase, TB_WAIT_LIMIT);  // once more, for the issued MMAs
    return false;
  }
  phase ^= 1u;
  tc::fence_after_sync();
  const uint32_t lane_addr = c.tmem + (uint32_t(((threadIdx.x >> 5) & 3) * 32) << 16);
  tab_drain<NMAX>(lane_addr, n, first);
  tc::fence_before_sync();
  __syncthreads();
  return true;
}

template <class S>
__device__ __forceinline__ void tab_end(const TabCta& c) {
  tc::fence_before_sync();
  __syncthreads();
  if ((threadIdx.x >> 5) == 0) tc::tmem_dealloc(c.tmem, S::TMEM_COLS);
}

// the S columns [cb, cb + 16) of accumulator acc of this thread's lane
template <int NMAX>
__device__ __forceinline__ void tab_read_sum(const TabCta& c, int acc, int cb, float* v) {
  const uint32_t lane_addr = c.tmem + (uint32_t(((threadIdx.x >> 5) & 3) * 32) << 16);
  tc::tmem_ld16(lane_addr + uint32_t(2 * NMAX + acc * NMAX + cb), v);
  tc::tmem_ld_wait();
}

__device__ __forceinline__ int round16(int x) { return (x + 15) & ~15; }

// raw table tile of the synthesis: the 32 units (quads) of one block and ring tile, each unit at a
// padded stride (unit + 16 bytes) so that lanes reading different units hit different banks
template <int NOPS>
struct SynthStg {
  static constexpr int UNIT = NOPS * TB_LB * 4;  // floats
  static constexpr int USTR = UNIT + 4;
  static constexpr uint32_t BYTES = 32u * USTR * 4u;
};

// ------------------------------------------------------------------ synthesis
// almT [nalm][B][NOPS] complex128 -> phase [R][mmax+1][B][NOPS] complex64 of the ring pairs
// [0, nrp) (table rings toff + i; north row i, south row R - 1 - i, R = 2 nrp - 1).
// grid.x = map group + G * (ring tile + T * m).  One CTA of 16 warps per SM: the table tiles of
// the next two blocks are in flight (bulk copies into the staging buffers) while a stage is split
// and multiplied; every thread has one operand task per stage.
template <int NOPS, int NMAX>
__global__ void __launch_bounds__(TM_THREADS, 1) tab_synth_kernel(const float* __restrict__ table,
                                                                   const int64_t* __restrict__ blockoff, int nquads,
                                                                   int toff, int nrp, int lmax, int mmax,
                                                                   const double2* __restrict__ almT,
                                                                   float2* __restrict__ phase, int B, int gsize,
                                                                   int ngroups, int ntiles, int spin_odd,
                                                                   int* __restrict__ err_flag) {
  using G = SynthStg<NOPS>;
  using S = TabSmem<NMAX, G::BYTES>;
  constexpr int NCOMP = NOPS;
  constexpr int UNIT = G::UNIT;
  extern __shared__ uint8_t tab_smem_raw[];
  int bid = blockIdx.x;
  const int grp = bid % ngroups; bid /= ngroups;
  const int tile = bid % ntiles;
  const int m = bid / ntiles;
  const int b0 = grp * gsize;
  const int gs = min(gsize, B - b0);
  const int ncols = 2 * NCOMP * gs;
  const int n = round16(ncols);
  const uint32_t idesc = tc::idesc_tf32(128, n, 0, 0);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  TabCta c = tab_begin<S>(tab_smem_raw);
  const int q0 = toff / 4 + tile * 32;  // first table quad of the tile
  const int nb = tab_nblocks(m, lmax);
  const int64_t base = alm_index(m, m, lmax);
  const int nhalf = NOPS == 1 ? 1 : 2;  // stages per table block
  const int nst = nb * nhalf;
  const int nvq = max(0, min(32, nquads - q0));  // units of the tile inside the table
  int issued = 0, waited = 0;  // blocks whose copies were issued / whose buffer wait completed (all threads)
  // bulk copies of block b's tile into staging buffer b & 1 (warp 0: lane q copies unit q)
  auto issue_block = [&](int b) {
    if (b >= nb) return;
    issued = b + 1;
    if (warp != 0) return;
    const uint32_t bar = c.mbar_full + 8u * uint32_t(b & 1);
    if (lane == 0) tc::mbar_arrive_expect_tx(bar, uint32_t(nvq) * UNIT * 4u);
    __syncwarp();  // the transaction count is expected before any unit lands
    if (lane < nvq) {
      const float* src = table + ((blockoff[m] + b) * int64_t(nquads) + q0 + lane) * UNIT;
      tc::bulk_g2s(c.sbase + S::stg(b & 1) + uint32_t(lane) * G::USTR * 4u, src, UNIT * 4u, bar);
    }
  };
  // ---- this thread's A task (the same every stage): warp = task (K chunk and accumulator), lane = quad
  int a_acc, a_pos0, a_comp;
  {
    const int t = warp;
    if (NOPS == 1) {
      a_acc = t >> 3; a_pos0 = a_acc * 32 + 4 * (t & 7); a_comp = 0;
    } else {
      a_comp = t >> 3;
      const int par = (t >> 2) & 1, g4 = t & 3;
      a_acc = a_comp == 0 ? par : 1 - par;
      a_pos0 = par * 32 + 4 * g4;  // + 16 h
    }
  }
  const int a_kk = NOPS == 1 ? 4 * (warp & 7) : 16 * (warp >> 3) + 4 * (warp & 3);
  const uint32_t a_oh = S::a(a_acc, a_kk >> 3, 0), a_ol = S::a(a_acc, a_kk >> 3, 1);
  const int a_kc = (a_kk >> 2) & 1;
  bool a_in[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int rt = 4 * (q0 + lane) + i;
    a_in[i] = rt >= toff && rt < toff + nrp && lane < nvq;
  }
  // ---- this thread's B tasks: spin 0: t = tid + 512 i (map j = t % gs, (acc, k4) = t / gs), 16 gs <= 1024;
  // spin s: t = tid < 256 (map j = t & 15, (acc, k4) = t >> 4)
  constexpr int BTS = NOPS == 1 ? 2 : 1;
  int b_j[BTS], b_acc[BTS], b_k4[BTS], b_lofs[BTS];
  bool b_v[BTS];
#pragma unroll
  for (int i2 = 0; i2 < BTS; ++i2) {
    const int t = tid + TM_THREADS * i2;
    if (NOPS == 1) {
      b_v[i2] = t < 16 * gs;
      const int j = b_v[i2] ? t % gs : 0, ak = b_v[i2] ? t / gs : 0;
      b_j[i2] = j; b_acc[i2] = ak >> 3; b_k4[i2] = ak & 7;
      b_lofs[i2] = 8 * b_k4[i2] + b_acc[i2];  // l = m + 64 b + b_lofs + 2 i
    } else {
      const int j = t & 15, ak = (t >> 4) & 15;
      b_v[i2] = t < 256 && j < gs;
      b_j[i2] = j; b_acc[i2] = ak >> 3; b_k4[i2] = ak & 7;
      const int comp = b_k4[i2] >> 2, g4 = b_k4[i2] & 3, par = comp == 0 ? b_acc[i2] : 1 - b_acc[i2];
      b_lofs[i2] = 2 * 4 * g4 + par;  // l = m + 64 b + 32 h + b_lofs + 2 i
    }
  }
  // alm of one stage in registers (FP32), loaded a stage ahead: spin 0 (re, im) of 4 l per task,
  // spin s G and C of 4 l
  float2 ab[BTS][2][4];
  auto load_alm = [&](int st) {
    const int b = st / nhalf, h = st % nhalf;
#pragma unroll
    for (int i2 = 0; i2 < BTS; ++i2) {
      const int l0 = m + TB_LB * b + 32 * h + b_lofs[i2];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int l = l0 + 2 * i;
        const bool v = b_v[i2] && l <= lmax;
        const int64_t o = ((base + (l - m)) * B + b0 + b_j[i2]) * NCOMP;
        const double2 x0 = v ? almT[o] : make_double2(0.0, 0.0);
        ab[i2][0][i] = make_float2(float(x0.x), float(x0.y));
        if (NOPS == 2) {
          const double2 x1 = v ? almT[o + 1] : make_double2(0.0, 0.0);
          ab[i2][1][i] = make_float2(float(x1.x), float(x1.y));
        }
      }
    }
  };
  // split and store the operands of stage st: A from the staged table tile, B from the registers
  auto store = [&](int st) {
    const int b = st / nhalf, h = st % nhalf;
    {
      const float* stg = reinterpret_cast<const float*>(c.smem + S::stg(b & 1));
      const float* u = stg + lane * G::USTR + (a_comp * TB_LB + a_pos0 + 16 * h) * 4;
      float4 v[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) v[i] = reinterpret_cast<const float4*>(u)[i];
      // ring 4 lane + i of the tile -> A row 32 i + lane; rings outside [toff, toff + nrp) are zero
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        float4 w;
        w.x = a_in[i] ? (&v[0].x)[i] : 0.f;
        w.y = a_in[i] ? (&v[1].x)[i] : 0.f;
        w.z = a_in[i] ? (&v[2].x)[i] : 0.f;
        w.w = a_in[i] ? (&v[3].x)[i] : 0.f;
        const uint32_t co = kcore_off(32 * i + lane, a_kc);
        st_split(c.smem, a_oh + co, a_ol + co, w);
      }
    }
#pragma unroll
    for (int i2 = 0; i2 < BTS; ++i2) {
      if (!b_v[i2]) continue;
      const int j = b_j[i2], acc = b_acc[i2], k4 = b_k4[i2];
      const int ks = k4 >> 1, kc = k4 & 1;
      if (NOPS == 1) {
        const float4 re = make_float4(ab[i2][0][0].x, ab[i2][0][1].x, ab[i2][0][2].x, ab[i2][0][3].x);
        const float4 im = make_float4(ab[i2][0][0].y, ab[i2][0][1].y, ab[i2][0][2].y, ab[i2][0][3].y);
        st_split(c.smem, S::b(acc, ks, 0) + kcore_off(j, kc), S::b(acc, ks, 1) + kcore_off(j, kc), re);
        st_split(c.smem, S::b(acc, ks, 0) + kcore_off(gs + j, kc), S::b(acc, ks, 1) + kcore_off(gs + j, kc), im);
      } else {
        // F+ rows take X = -(G, C) (even spin) or Y = (C.im, -C.re, -G.im, G.re); F- rows the other one
        const int comp = k4 >> 2;
        const bool use_x = (comp == 0) != (spin_odd != 0);
        float4 pt[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const float2 Gv = ab[i2][0][i], Cv = ab[i2][1][i];
          float p0, p1, p2, p3;
          if (use_x) { p0 = -Gv.x; p1 = -Gv.y; p2 = -Cv.x; p3 = -Cv.y; }
          else { p0 = Cv.y; p1 = -Cv.x; p2 = -Gv.y; p3 = Gv.x; }
          (&pt[0].x)[i] = p0; (&pt[1].x)[i] = p1; (&pt[2].x)[i] = p2; (&pt[3].x)[i] = p3;
        }
#pragma unroll
        for (int part = 0; part < 4; ++part) {
          const int row = part * gs + j;
          st_split(c.smem, S::b(acc, ks, 0) + kcore_off(row, kc), S::b(acc, ks, 1) + kcore_off(row, kc), pt[part]);
        }
      }
    }
  };
  uint32_t ph_mma = 0;
  bool ok = true;
  issue_block(0);
  issue_block(1);
  load_alm(0);
  for (int st = 0; st < nst; ++st) {
    const int b = st / nhalf, h = st % nhalf;
    if (h == 0) {
      if (!tab_wait(c.mbar_full + 8u * uint32_t(b & 1), uint32_t(b >> 1) & 1u, err_flag)) {
        ok = false;
        break;
      }
      waited = b + 1;
    }
    store(st);
    tab_issue_stage<S, NMAX>(c, idesc);
    // the staged tile of block b has been read (barrier inside tab_issue_stage): refill its buffer
    if (h == nhalf - 1) issue_block(b + 2);
    if (st + 1 < nst) load_alm(st + 1);
    ok = tab_finish_stage<NMAX>(c, n, st == 0, ph_mma, err_flag);
    if (!ok) break;
  }
  if (ok) {
    // epilogue.  TMEM lane tl = 32 lq + q <-> ring 4 q + lq of the tile (lq = warp & 3).  The sums go
    // through shared memory (free now: every MMA and copy has completed) as rows [north/south][tl]
    // [map][part], then every ring's row of gs maps is written with coalesced stores
    constexpr int RS = NMAX + 1;  // row stride (floats): consecutive lanes in consecutive banks
    static_assert(2 * 128 * RS * 4 <= int(S::MISC_OFF), "epilogue rows exceed the free shared memory");
    float* rows = reinterpret_cast<float*>(c.smem);
    const int lq = warp & 3, cs = warp >> 2;
    const int tl = 32 * lq + lane;
#pragma unroll 1
    for (int cb = 16 * cs; cb < n; cb += 64) {
      float s0[16], s1[16];
      tab_read_sum<NMAX>(c, 0, cb, s0);
      tab_read_sum<NMAX>(c, 1, cb, s1);
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const int col = cb + q;
        if (col >= ncols) break;
        const int part = col / gs, j = col % gs;
        const int pos = j * 2 * NCOMP + part;
        rows[tl * RS + pos] = s0[q] + s1[q];
        rows[(128 + tl) * RS + pos] = s0[q] - s1[q];
      }
    }
    __syncthreads();
    const int R = 2 * nrp - 1;
#pragma unroll 1
    for (int row = warp; row < 256; row += TM_THREADS / 32) {
      const int ns = row >> 7, t = row & 127;
      const int rt = 4 * q0 + 4 * (t & 31) + (t >> 5);  // table ring of TMEM lane t
      const int i = rt - toff;                          // ring pair of the plan
      if (rt < toff || i >= nrp) continue;
      const int ring = ns == 0 ? i : R - 1 - i;
      if (ns == 1 && ring == i) continue;  // the equator has no south ring
      float* dst = reinterpret_cast<float*>(phase + ((int64_t(ring) * (mmax + 1) + m) * B + b0) * NCOMP);
      const float* src = rows + row * RS;
      for (int pos = lane; pos < ncols; pos += 32) dst[pos] = src[pos];
    }
  } else if (threadIdx.x == 0) {
    // bulk copies still in flight land in this CTA's shared memory: wait for them (bounded) before exit
    for (int k = waited; k < issued; ++k)
      tc::mbar_wait_bounded(c.mbar_full + 8u * uint32_t(k & 1), uint32_t(k >> 1) & 1u, TB_WAIT_LIMIT);
  }
  tab_end<S>(c);
}

// raw table tile of one adjoint stage: for each of the 4 blocks, the RSTAGE / 4 consecutive units
// (spin s: followed by the phases of the stage's rings, [north/south][ring][map] complex64 pairs
// with a row stride of PH_MAPS maps)
template <int NOPS>
struct AdjStg {
  static constexpr int UNIT = NOPS * TB_LB * 4;
  static constexpr int NQ = NOPS == 1 ? 8 : 4;  // quads per stage
  static constexpr uint32_t BLK_BYTES = uint32_t(NQ) * UNIT * 4u;
  static constexpr uint32_t TAB_BYTES = 4u * BLK_BYTES;
  static constexpr int PH_MAPS = 32;  // maps per group (spin s)
  static constexpr uint32_t PH_BYTES = NOPS == 2 ? 2u * 4u * NQ * PH_MAPS * 16u : 0u;
  static constexpr uint32_t BYTES = TAB_BYTES + PH_BYTES;
};

// ------------------------------------------------------------------ adjoint
// phase [R][mmax+1][B][NOPS] complex64 of ring pairs [0, nrp) -> alm of map b at alm + b * out_stride
// ([NOPS][nalm] complex128, times scale and lscale[comp][idx] when given), for the maps [b0, b0 + gs)
// of each group.  grid.x = map group + G * (entry of the (m, first block) work list)
template <int NOPS, int NMAX>
__global__ void __launch_bounds__(TM_THREADS, 1) tab_adj_kernel(const float* __restrict__ table,
                                                                 const int64_t* __restrict__ blockoff, int nquads,
                                                                 int toff, int nrp, int lmax, int mmax,
                                                                 const float2* __restrict__ phase,
                                                                 double2* __restrict__ alm, int B, int gsize,
                                                                 int ngroups, const int2* __restrict__ work,
                                                                 int64_t nalm, double scale, int spin_odd,
                                                                 int64_t out_stride,
                                                                 const double* __restrict__ lscale,
                                                                 int* __restrict__ err_flag) {
  using G = AdjStg<NOPS>;
  using S = TabSmem<NMAX, G::BYTES>;
  constexpr int NCOMP = NOPS;
  constexpr int UNIT = G::UNIT;
  constexpr int RSTAGE = 4 * G::NQ;  // table rings per stage
  constexpr int NQ = G::NQ;
  extern __shared__ uint8_t tab_smem_raw[];
  int bid = blockIdx.x;
  const int grp = bid % ngroups; bid /= ngroups;
  const int2 wk = work[bid];  // (m, first block of the group of 4)
  const int m = wk.x, bb = wk.y;
  const int b0 = grp * gsize;
  const int gs = min(gsize, B - b0);
  const int ncols = 2 * NCOMP * gs;
  const int n = round16(ncols);
  const uint32_t idesc = tc::idesc_tf32(128, n, 0, 0);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  TabCta c = tab_begin<S>(tab_smem_raw);
  const int nb = tab_nblocks(m, lmax);
  const int R = 2 * nrp - 1;
  const int rt_begin = toff & ~3, rt_end = toff + nrp;
  const int nstages = (rt_end - rt_begin + RSTAGE - 1) / RSTAGE;
  int issued = 0, waited = 0;  // stages whose copies were issued / whose buffer wait completed (all threads)
  // bulk copies of stage st's units into staging buffer st & 1 (thread 0)
  // bulk copies of stage st's units (and, spin s, of its phase rows) into staging buffer st & 1
  // (warp 0: lane 0 the table units, lane r the phase rows of ring r of the stage)
  auto issue_stage_copy = [&](int st) {
    if (st >= nstages) return;
    issued = st + 1;
    if (warp != 0) return;
    const int rs0 = rt_begin + st * RSTAGE;
    const int qs = rs0 / 4;
    const int nvq = max(0, min(NQ, nquads - qs));
    int nblk = 0;
    for (int blk = 0; blk < 4; ++blk) nblk += (bb + blk < nb);
    uint32_t tx = uint32_t(nblk * nvq) * UNIT * 4u;
    // spin s: ring rs0 + r (r = lane < RSTAGE) has a north row when it is a ring of the plan, and a
    // south row unless it is the equator
    const int ip = rs0 + lane - toff;
    const bool ph_n = NOPS == 2 && lane < RSTAGE && ip >= 0 && ip < nrp;
    const bool ph_s = ph_n && R - 1 - ip != ip;
    const uint32_t row_bytes = uint32_t(gs) * 16u;
    if (NOPS == 2) {
      uint32_t rows = uint32_t(ph_n) + uint32_t(ph_s);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) rows += __shfl_xor_sync(0xffffffffu, rows, o);
      tx += rows * row_bytes;
    }
    const uint32_t bar = c.mbar_full + 8u * uint32_t(st & 1);
    const uint32_t dst = c.sbase + S::stg(st & 1);
    if (lane == 0) {
      tc::mbar_arrive_expect_tx(bar, tx);
      for (int blk = 0; blk < 4; ++blk) {
        if (bb + blk >= nb || nvq == 0) continue;
        const float* src = table + ((blockoff[m] + bb + blk) * int64_t(nquads) + qs) * UNIT;
        tc::bulk_g2s(dst + uint32_t(blk) * G::BLK_BYTES, src, uint32_t(nvq) * UNIT * 4u, bar);
      }
    }
    if (NOPS == 2) {
      __syncwarp();  // the transaction count is expected before any phase row lands
      const uint32_t pd = dst + G::TAB_BYTES + uint32_t(lane) * G::PH_MAPS * 16u;
      if (ph_n)
        tc::bulk_g2s(pd, phase + ((int64_t(ip) * (mmax + 1) + m) * B + b0) * NCOMP, row_bytes, bar);
      if (ph_s)
        tc::bulk_g2s(pd + uint32_t(RSTAGE) * G::PH_MAPS * 16u,
                     phase + ((int64_t(R - 1 - ip) * (mmax + 1) + m) * B + b0) * NCOMP, row_bytes, bar);
    }
  };
  // ---- A tasks: combination t = warp + 16 it (quad, comp, block, acc), lane = position in the parity half
  constexpr int NT = 2 * 4 * NOPS * NQ;  // 64
  constexpr int NA = NT / (TM_THREADS / 32);
  // ---- B tasks.  spin 0: t = tid (map j = t % gs, quad qd = t / gs), NQ gs <= 512, phases loaded to
  // registers a stage ahead.  spin s: t = tid (sub = t & 3 -> (acc, comp), map j = (t >> 2) % gs,
  // quad qd = (t >> 2) / gs), NQ gs <= 128, phases read from the staged rows
  const int p_t = NOPS == 1 ? tid : tid >> 2;
  const bool p_v = p_t < NQ * gs;
  const int p_j = p_v ? p_t % gs : 0, p_qd = p_v ? p_t / gs : 0;
  float2 pn[4], pv[4];
  auto load_phase = [&](int st) {
    if (NOPS != 1) return;
    const int rs0 = rt_begin + st * RSTAGE;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int rt = rs0 + 4 * p_qd + i;
      const int ip = rt - toff;
      const bool in = p_v && rt >= toff && ip < nrp;
      const int rsth = R - 1 - ip;
      pn[i] = in ? phase[(int64_t(ip) * (mmax + 1) + m) * B + b0 + p_j] : make_float2(0.f, 0.f);
      pv[i] = (in && rsth != ip) ? phase[(int64_t(rsth) * (mmax + 1) + m) * B + b0 + p_j] : make_float2(0.f, 0.f);
    }
  };
  auto store = [&](int st) {
    const int rs0 = rt_begin + st * RSTAGE;
    const float* stg = reinterpret_cast<const float*>(c.smem + S::stg(st & 1));
#pragma unroll
    for (int it = 0; it < NA; ++it) {
      const int t = warp + (TM_THREADS / 32) * it;
      const int qd = t % NQ;
      int r = t / NQ;
      const int comp = r % NOPS; r /= NOPS;
      const int blk = r % 4;
      const int acc = r / 4;
      const int b = bb + blk;
      const int qg = rs0 / 4 + qd;
      float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
      if (b < nb && qg < nquads) {
        v = *reinterpret_cast<const float4*>(stg + blk * (G::BLK_BYTES / 4) + qd * UNIT +
                                             (comp * TB_LB + acc * 32 + lane) * 4);
        // rings outside [toff, toff + nrp) contribute nothing
        const int r0 = 4 * qg;
        if (r0 < toff || r0 + 3 >= rt_end) {
          if (r0 + 0 < toff || r0 + 0 >= rt_end) v.x = 0.f;
          if (r0 + 1 < toff || r0 + 1 >= rt_end) v.y = 0.f;
          if (r0 + 2 < toff || r0 + 2 >= rt_end) v.z = 0.f;
          if (r0 + 3 < toff || r0 + 3 >= rt_end) v.w = 0.f;
        }
      }
      const int kk = comp * 16 + 4 * qd;  // K index of the chunk (spin 0: comp = 0, qd < 8)
      const int ks = kk >> 3, kc = (kk >> 2) & 1;
      const int row = blk * 32 + lane;
      st_split(c.smem, S::a(acc, ks, 0) + kcore_off(row, kc), S::a(acc, ks, 1) + kcore_off(row, kc), v);
    }
    if (p_v && NOPS == 1) {
      const int j = p_j, qd = p_qd;
      // ring sums (combo 0: N + S) and differences (combo 1: N - S) of 4 rings
      float4 cre[2], cim[2];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        (&cre[0].x)[i] = pn[i].x + pv[i].x;
        (&cim[0].x)[i] = pn[i].y + pv[i].y;
        (&cre[1].x)[i] = pn[i].x - pv[i].x;
        (&cim[1].x)[i] = pn[i].y - pv[i].y;
      }
      const int kk = 4 * qd, ks = kk >> 3, kc = (kk >> 2) & 1;
#pragma unroll
      for (int acc = 0; acc < 2; ++acc) {
        st_split(c.smem, S::b(acc, ks, 0) + kcore_off(j, kc), S::b(acc, ks, 1) + kcore_off(j, kc), cre[acc]);
        st_split(c.smem, S::b(acc, ks, 0) + kcore_off(gs + j, kc), S::b(acc, ks, 1) + kcore_off(gs + j, kc),
                 cim[acc]);
      }
    } else if (p_v) {
      // columns (G.re, G.im, C.re, C.im); combo k (0: N + S, 1: N - S) of the rings' (Q, U):
      // Xa(k) = (-Q.re, -Q.im, -U.re, -U.im), Ya(k) = (U.im, -U.re, -Q.im, Q.re)
      // even spin: F+ rows Xa(acc), F- rows Ya(1 - acc); odd spin: F+ rows Ya(acc), F- rows Xa(1 - acc)
      const int j = p_j, qd = p_qd;
      const int acc = (tid >> 1) & 1, comp = tid & 1;
      const int k = comp == 0 ? acc : 1 - acc;
      const bool use_x = (comp == 0) != (spin_odd != 0);
      const float4* ph = reinterpret_cast<const float4*>(c.smem + S::stg(st & 1) + G::TAB_BYTES);
      float4 p[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int r = 4 * qd + i;  // ring of the stage
        const int ip = rs0 + r - toff;
        const bool in = ip >= 0 && ip < nrp;
        const bool hs = in && R - 1 - ip != ip;
        const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
        const float4 nv = in ? ph[r * G::PH_MAPS + j] : z;
        const float4 sv = hs ? ph[(RSTAGE + r) * G::PH_MAPS + j] : z;
        const float4 cv = k == 0 ? make_float4(nv.x + sv.x, nv.y + sv.y, nv.z + sv.z, nv.w + sv.w)
                                 : make_float4(nv.x - sv.x, nv.y - sv.y, nv.z - sv.z, nv.w - sv.w);
        // cv = (Q.re, Q.im, U.re, U.im) of ring i
        if (use_x) {
          (&p[0].x)[i] = -cv.x; (&p[1].x)[i] = -cv.y; (&p[2].x)[i] = -cv.z; (&p[3].x)[i] = -cv.w;
        } else {
          (&p[0].x)[i] = cv.w; (&p[1].x)[i] = -cv.z; (&p[2].x)[i] = -cv.y; (&p[3].x)[i] = cv.x;
        }
      }
      const int kk = comp * 16 + 4 * qd, ks = kk >> 3, kc = (kk >> 2) & 1;
#pragma unroll
      for (int part = 0; part < 4; ++part) {
        const int row = part * gs + j;
        st_split(c.smem, S::b(acc, ks, 0) + kcore_off(row, kc), S::b(acc, ks, 1) + kcore_off(row, kc), p[part]);
      }
    }
  };
  uint32_t ph_mma = 0;
  bool ok = true;
  issue_stage_copy(0);
  issue_stage_copy(1);
  load_phase(0);
  for (int st = 0; st < nstages; ++st) {
    if (!tab_wait(c.mbar_full + 8u * uint32_t(st & 1), uint32_t(st >> 1) & 1u, err_flag)) {
      ok = false;
      break;
    }
    waited = st + 1;
    store(st);
    tab_issue_stage<S, NMAX>(c, idesc);
    issue_stage_copy(st + 2);  // staging buffer st & 1 has been read (barrier inside tab_issue_stage)
    if (st + 1 < nstages) load_phase(st + 1);
    ok = tab_finish_stage<NMAX>(c, n, st == 0, ph_mma, err_flag);
    if (!ok) break;
  }
  if (ok) {
    // epilogue: TMEM lane = A row = blk * 32 + j (blk = warp & 3); accumulator acc is
    // l = tab_l(m, bb + blk, acc * 32 + j); the four warps of a lane quarter take every fourth column chunk
    const int blk = warp & 3, cs = warp >> 2, j = lane;
    const int b = bb + blk;
#pragma unroll 1
    for (int acc = 0; acc < 2; ++acc) {
      const int l = tab_l(m, b, acc * 32 + j);
      const bool in = b < nb && l <= lmax;
      const int64_t idx = alm_index(l, m, lmax);
#pragma unroll 1
      for (int cb = 16 * cs; cb < n; cb += 64) {
        float s[16];
        tab_read_sum<NMAX>(c, acc, cb, s);
        if (!in) continue;
        // columns come in (re, im) pairs of one complex value only when gs is even; write parts one by one
#pragma unroll
        for (int q = 0; q < 16; ++q) {
          const int col = cb + q;
          if (col >= ncols) break;
          const int part = col / gs, jm = col % gs;
          const int comp = part >> 1;
          const double f = lscale ? scale * lscale[int64_t(comp) * nalm + idx] : scale;
          double* dst = reinterpret_cast<double*>(alm + int64_t(b0 + jm) * out_stride + int64_t(comp) * nalm + idx) +
                        (part & 1);
          *dst = double(s[q]) * f;
        }
      }
    }
  } else if (threadIdx.x == 0) {
    for (int k = waited; k < issued; ++k)
      tc::mbar_wait_bounded(c.mbar_full + 8u * uint32_t(k & 1), uint32_t(k >> 1) & 1u, TB_WAIT_LIMIT);
  }
  tab_end<S>(c);
}

// ------------------------------------------------------------------ host side
namespace {
// the dynamic shared-memory opt-in is per device and function; setting it before every launch
// keeps it right on whichever device the caller made current
int set_smem_attr(const void* fn, int bytes) {
  return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) == cudaSuccess ? PS_OK
                                                                                                       : PS_ERR_CUDA;
}
}  // namespace

int64_t tab_total_blocks(int lmax, int mmax) {
  int64_t t = 0;
  for (int m = 0; m <= mmax; ++m) t += tab_nblocks(m, lmax);
  return t;
}

void tab_blockoff(int lmax, int mmax, std::vector<int64_t>& off) {
  off.resize(mmax + 2);
  int64_t t = 0;
  for (int m = 0; m <= mmax; ++m) { off[m] = t; t += tab_nblocks(m, lmax); }
  off[mmax + 1] = t;
}

int tab_quads(int Rh) { return ((Rh + TB_TILE - 1) / TB_TILE) * TB_TILE / 4; }

size_t tab_bytes(int Rh, int lmax, int mmax, int spin) {
  return size_t(tab_total_blocks(lmax, mmax)) * size_t(tab_quads(Rh)) * size_t(spin == 0 ? 1 : 2) * TB_LB * 4 *
         sizeof(float);
}

int launch_tab_gen(const Plan& P, int spin, const int64_t* d_blockoff, float* table, cudaStream_t st) {
  const int nquads = tab_quads(P.Rh);
  dim3 grid(nquads * 4 / TB_TILE, P.mmax + 1);
  if (spin == 0) {
    const int smem = 32 * (1 * TB_LB * 4 + 4) * sizeof(float);
    if (set_smem_attr((const void*)tab_gen_kernel<1>, smem)) return PS_ERR_CUDA;
    tab_gen_kernel<1><<<grid, TB_THREADS, smem, st>>>(P.d_rings, P.d_mnorm0, nullptr, P.Rh, P.lmax, 0, d_blockoff,
                                                      nquads, table);
  } else {
    if (!P.d_seed[spin]) return PS_ERR_INVALID;
    const int smem = 32 * (2 * TB_LB * 4 + 4) * sizeof(float);
    if (set_smem_attr((const void*)tab_gen_kernel<2>, smem)) return PS_ERR_CUDA;
    tab_gen_kernel<2><<<grid, TB_THREADS, smem, st>>>(P.d_rings, nullptr, P.d_seed[spin], P.Rh, P.lmax, spin,
                                                      d_blockoff, nquads, table);
  }
  PS_LAUNCH_CHECK();
  return PS_OK;
}

// maps per group: as many as fit the nmax columns of an accumulator, spread evenly over the groups
static int tab_group_size(int B, int spin, int nmax, int& ngroups) {
  const int cap = spin == 0 ? nmax / 2 : nmax / 4;
  ngroups = (B + cap - 1) / cap;
  return (B + ngroups - 1) / ngroups;
}

// The table of ring pairs [toff, toff + nrp) of a plan with Rh_table ring pairs (a band plan reads its
// parent's table at an offset).
int launch_tab_synth(const Plan& P, const float* table, const int64_t* d_blockoff, int Rh_table, int toff,
                     const double2* almT, float2* phase, int B, int spin, int* err_flag, cudaStream_t st) {
  const double flops = double(spin == 0 ? 4 : 16) * double(P.Rh) * double(P.nalm) * B;
  const double bytes = double(tab_bytes(Rh_table, P.lmax, P.mmax, spin)) * double(P.Rh) / double(Rh_table) +
                       double(B) * (spin == 0 ? 1 : 2) * (16.0 * P.nalm + 8.0 * P.R * (P.mmax + 1));
  StatScope sc(PS_K_LEG_SYNTH, flops, bytes, st);
  // 128 columns per accumulator for spin 0 (up to 64 maps per pass over the table), 64 for spin s
  // (16 maps; its staged tiles are twice as large, which leaves shared memory for no more)
  const int nmax = spin == 0 ? 128 : 64;
  int ngroups = 1;
  const int gsize = tab_group_size(B, spin, nmax, ngroups);
  const int ntiles = ((toff & 3) + P.Rh + TB_TILE - 1) / TB_TILE;
  const int nquads = tab_quads(Rh_table);
  const int64_t nblk = int64_t(ngroups) * ntiles * (P.mmax + 1);
  if (nblk > 0x7fffffff) return PS_ERR_UNSUPPORTED;
  if (spin == 0) {
    const int smem = int(TabSmem<128, SynthStg<1>::BYTES>::DYN);
    if (set_smem_attr((const void*)tab_synth_kernel<1, 128>, smem)) return PS_ERR_CUDA;
    tab_synth_kernel<1, 128><<<unsigned(nblk), TM_THREADS, smem, st>>>(table, d_blockoff, nquads, toff, P.Rh, P.lmax,
                                                                       P.mmax, almT, phase, B, gsize, ngroups, ntiles,
                                                                       0, err_flag);
  } else {
    const int smem = int(TabSmem<64, SynthStg<2>::BYTES>::DYN);
    if (set_smem_attr((const void*)tab_synth_kernel<2, 64>, smem)) return PS_ERR_CUDA;
    tab_synth_kernel<2, 64><<<unsigned(nblk), TM_THREADS, smem, st>>>(table, d_blockoff, nquads, toff, P.Rh, P.lmax,
                                                                      P.mmax, almT, phase, B, gsize, ngroups, ntiles,
                                                                      spin & 1, err_flag);
  }
  PS_LAUNCH_CHECK();
  return PS_OK;
}

// work list of the adjoint: (m, first block) of every group of 4 blocks, heaviest orders first
void tab_adj_work(int lmax, int mmax, std::vector<int2>& work) {
  work.clear();
  for (int m = 0; m <= mmax; ++m)
    for (int b = 0; b < tab_nblocks(m, lmax); b += 4) work.push_back(make_int2(m, b));
}

// alm (B maps) at alm + b * out_stride (complex elements; ncomp * nalm for a contiguous batch), each value
// times scale and, when lscale is given, lscale[comp][idx]
int launch_tab_adj(const Plan& P, const float* table, const int64_t* d_blockoff, const int2* d_work, int nwork,
                   int Rh_table, int toff, const float2* phase, double2* alm, int B, int spin, double scale,
                   int64_t out_stride, const double* lscale, int* err_flag, cudaStream_t st) {
  const double flops = double(spin == 0 ? 4 : 16) * double(P.Rh) * double(P.nalm) * B;
  const double bytes = double(tab_bytes(Rh_table, P.lmax, P.mmax, spin)) * double(P.Rh) / double(Rh_table) +
                       double(B) * (spin == 0 ? 1 : 2) * (16.0 * P.nalm + 8.0 * P.R * (P.mmax + 1));
  StatScope sc(PS_K_LEG_ADJOINT, flops, bytes, st);
  // 128 columns per accumulator: up to 64 maps of spin 0 or 32 of spin s per pass over the table
  constexpr int nmax = 128;
  int ngroups = 1;
  const int gsize = tab_group_size(B, spin, nmax, ngroups);
  const int nquads = tab_quads(Rh_table);
  const int64_t nblk = int64_t(ngroups) * nwork;
  if (nblk > 0x7fffffff) return PS_ERR_UNSUPPORTED;
  // spin s phase rows are staged by bulk copies, which start on 16-byte boundaries
  if (spin != 0 && (reinterpret_cast<uintptr_t>(phase) & 15u)) return PS_ERR_INVALID;
  if (spin == 0) {
    const int smem = int(TabSmem<nmax, AdjStg<1>::BYTES>::DYN);
    if (set_smem_attr((const void*)tab_adj_kernel<1, nmax>, smem)) return PS_ERR_CUDA;
    tab_adj_kernel<1, nmax><<<unsigned(nblk), TM_THREADS, smem, st>>>(table, d_blockoff, nquads, toff, P.Rh, P.lmax,
                                                                      P.mmax, phase, alm, B, gsize, ngroups, d_work,
                                                                      P.nalm, scale, 0, out_stride, lscale, err_flag);
  } else {
    const int smem = int(TabSmem<nmax, AdjStg<2>::BYTES>::DYN);
    if (set_smem_attr((const void*)tab_adj_kernel<2, nmax>, smem)) return PS_ERR_CUDA;
    tab_adj_kernel<2, nmax><<<unsigned(nblk), TM_THREADS, smem, st>>>(table, d_blockoff, nquads, toff, P.Rh, P.lmax,
                                                                      P.mmax, phase, alm, B, gsize, ngroups, d_work,
                                                                      P.nalm, scale, spin & 1, out_stride, lscale,
                                                                      err_flag);
  }
  PS_LAUNCH_CHECK();
  return PS_OK;
}

}  // namespace ps
