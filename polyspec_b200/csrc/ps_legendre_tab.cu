// Table-driven mixed-precision Legendre stages on the tensor cores (tcgen05,
// kind::tf32, accumulators in TMEM).
//
// The normalised Legendre values of a plan do not depend on the data, so for
// a mixed-precision plan they can be computed once (FP64 recurrence with the
// scaled seeds of the on-the-fly kernels, rounded to FP32) and kept in HBM in
// the order in which the two GEMMs below consume them.  Each transform then
// streams the table instead of re-running the recurrence for every group of
// maps: at Nside 1024, lmax 2048 the spin-0 table is 17.7 GB and the spin-s
// table (F+ and F-) 35.4 GB, read once per transform of up to 32 (spin 0) or
// 16 (spin s) maps per map group.
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
// FP32 adds by the four epilogue warps).  TMEM: D[2 accumulators][64 columns]
// and S[2][64], 256 columns per CTA, two CTAs per SM.
//
// Columns of D are (part, map) with the part index outermost: spin 0
// (re, im) of the complex value, spin s four real parts; map group g of up
// to 32 (spin 0) or 16 (spin s) maps.  N = the used columns rounded up to 16.
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
constexpr int TB_NMAX = 64;      // D columns per accumulator
constexpr int TB_THREADS = 128;
constexpr uint32_t TB_WAIT_LIMIT = 1u << 24;
constexpr uint32_t TB_TMEM_COLS = 256;

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

// shared-memory plan of both GEMMs: A[acc][kstep][hi/lo] 4 KB each, B[acc][kstep][hi/lo] NMAX x 32 B each
struct TabSmem {
  static constexpr int KS = 4;  // K steps (of 8) per accumulator and stage
  static constexpr uint32_t A_TILE = TB_TILE * 32;
  static constexpr uint32_t B_TILE = TB_NMAX * 32;
  static constexpr uint32_t B_OFF = 2 * KS * 2 * A_TILE;
  static constexpr uint32_t MISC_OFF = B_OFF + 2 * KS * 2 * B_TILE;
  static constexpr uint32_t DYN = MISC_OFF + 64 + 1024;
  __device__ static uint32_t a(int acc, int ks, int hl) { return ((acc * KS + ks) * 2 + hl) * A_TILE; }
  __device__ static uint32_t b(int acc, int ks, int hl) { return B_OFF + ((acc * KS + ks) * 2 + hl) * B_TILE; }
};

// one stage's MMAs: 2 accumulators x 4 K steps x (hi.hi + hi.lo + lo.hi), D fresh per stage
__device__ __forceinline__ void tab_issue(uint32_t sbase, uint32_t tmem, uint32_t idesc) {
#pragma unroll
  for (int acc = 0; acc < 2; ++acc) {
    const uint32_t d = tmem + uint32_t(acc * TB_NMAX);
#pragma unroll
    for (int ks = 0; ks < TabSmem::KS; ++ks) {
      const uint64_t ah = kdesc(sbase + TabSmem::a(acc, ks, 0)), al = kdesc(sbase + TabSmem::a(acc, ks, 1));
      const uint64_t bh = kdesc(sbase + TabSmem::b(acc, ks, 0)), bl = kdesc(sbase + TabSmem::b(acc, ks, 1));
      tc::mma_tf32(d, ah, bh, idesc, ks > 0 ? 1u : 0u);
      tc::mma_tf32(d, ah, bl, idesc, 1u);
      tc::mma_tf32(d, al, bh, idesc, 1u);
    }
  }
}

// S += D for this thread's TMEM lane (first stage: S = D), columns [0, n) of both accumulators;
// the four loads of a column chunk (D and S of both accumulators) share one wait
__device__ __forceinline__ void tab_drain(uint32_t lane_addr, int n, bool first) {
#pragma unroll 1
  for (int cb = 0; cb < n; cb += 16) {
    float d0[16], d1[16], s0[16], s1[16];
    const uint32_t dc0 = lane_addr + uint32_t(cb), dc1 = lane_addr + uint32_t(TB_NMAX + cb);
    const uint32_t sc0 = lane_addr + uint32_t(2 * TB_NMAX + cb), sc1 = lane_addr + uint32_t(3 * TB_NMAX + cb);
    tc::tmem_ld16(dc0, d0);
    tc::tmem_ld16(dc1, d1);
    if (!first) {
      tc::tmem_ld16(sc0, s0);
      tc::tmem_ld16(sc1, s1);
    }
    tc::tmem_ld_wait();
    if (!first) {
#pragma unroll
      for (int q = 0; q < 16; ++q) { d0[q] += s0[q]; d1[q] += s1[q]; }
    }
    tmem_st16(sc0, d0);
    tmem_st16(sc1, d1);
  }
  tmem_st_wait();
}

// CTA prologue / epilogue shared by both GEMMs
struct TabCta {
  uint8_t* smem;
  uint32_t sbase;
  uint64_t* mbar;
  uint32_t tmem;
};

__device__ __forceinline__ TabCta tab_begin(uint8_t* smem_raw) {
  TabCta c;
  c.smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  c.sbase = tc::smem_u32(c.smem);
  c.mbar = reinterpret_cast<uint64_t*>(c.smem + TabSmem::MISC_OFF);
  uint32_t* slot = reinterpret_cast<uint32_t*>(c.smem + TabSmem::MISC_OFF + 16);
  if ((threadIdx.x >> 5) == 0) {
    tc::tmem_alloc(tc::smem_u32(slot), TB_TMEM_COLS);
    tc::tmem_relinquish();
  }
  if (threadIdx.x == 0) tc::mbar_init(tc::smem_u32(c.mbar), 1);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  c.tmem = *slot;
  return c;
}

// issue the stage's MMAs (thread 0) once every thread's operand stores are in shared memory
__device__ __forceinline__ void tab_issue_stage(const TabCta& c, uint32_t idesc) {
  tc::fence_proxy_async();
  __syncthreads();
  if (threadIdx.x == 0) {
    tc::fence_after_sync();
    tab_issue(c.sbase, c.tmem, idesc);
    tc::mma_commit(tc::smem_u32(c.mbar));
  }
}

// wait for the stage's MMAs and drain D into S; returns false (and raises the error flag) when
// the wait expires.  After it returns true the operand tiles may be overwritten.
__device__ __forceinline__ bool tab_finish_stage(const TabCta& c, int n, bool first, uint32_t& phase,
                                                 int* err_flag) {
  const bool ok = __syncthreads_and(tc::mbar_wait_bounded(tc::smem_u32(c.mbar), phase, TB_WAIT_LIMIT));
  if (!ok) {
    if (threadIdx.x == 0) atomicExch(err_flag, 1);
    tc::mbar_wait_bounded(tc::smem_u32(c.mbar), phase, TB_WAIT_LIMIT);
    return false;
  }
  phase ^= 1u;
  tc::fence_after_sync();
  const uint32_t lane_addr = c.tmem + (uint32_t((threadIdx.x >> 5) * 32) << 16);
  tab_drain(lane_addr, n, first);
  tc::fence_before_sync();
  __syncthreads();
  return true;
}

__device__ __forceinline__ void tab_end(const TabCta& c) {
  tc::fence_before_sync();
  __syncthreads();
  if ((threadIdx.x >> 5) == 0) tc::tmem_dealloc(c.tmem, TB_TMEM_COLS);
}

// the S columns [cb, cb + 16) of accumulator acc of this thread's lane
__device__ __forceinline__ void tab_read_sum(const TabCta& c, int acc, int cb, float* v) {
  const uint32_t lane_addr = c.tmem + (uint32_t((threadIdx.x >> 5) * 32) << 16);
  tc::tmem_ld16(lane_addr + uint32_t(2 * TB_NMAX + acc * TB_NMAX + cb), v);
  tc::tmem_ld_wait();
}

__device__ __forceinline__ int round16(int x) { return (x + 15) & ~15; }

// ------------------------------------------------------------------ synthesis
// almT [nalm][B][NCOMP] complex128 -> phase [R][mmax+1][B][NCOMP] complex64 of the ring pairs
// [0, nrp) (table rings toff + i; north row i, south row R - 1 - i, R = 2 nrp - 1).
// grid.x = map group + G * (ring tile + T * m)
template <int NOPS>
__global__ void __launch_bounds__(TB_THREADS, 2) tab_synth_kernel(const float* __restrict__ table,
                                                                   const int64_t* __restrict__ blockoff, int nquads,
                                                                   int toff, int nrp, int lmax, int mmax,
                                                                   const double2* __restrict__ almT,
                                                                   float2* __restrict__ phase, int B, int gsize,
                                                                   int ngroups, int ntiles, int spin_odd,
                                                                   int* __restrict__ err_flag) {
  constexpr int NCOMP = NOPS;
  constexpr int UNIT = NOPS * TB_LB * 4;
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
  TabCta c = tab_begin(tab_smem_raw);
  const int q0 = toff / 4 + tile * 32;  // first table quad of the tile
  const int nb = tab_nblocks(m, lmax);
  const int64_t base = alm_index(m, m, lmax);
  const int nhalf = NOPS == 1 ? 1 : 2;  // stages per table block
  const int nst = nb * nhalf;
  // Raw operands of one stage, held in registers from the global loads to the split and the
  // shared-memory stores, so that stage s + 1 is in flight while the MMAs of stage s run.
  // A: 4 tasks of a 4 (ring) x 4 (K) block (lane = quad, task t = warp + 4 it).
  // B: spin 0: 4 tasks (map lane, acc, k4) x 4 l of a_lm; spin s: 2 tasks (map lane & 15) x 4 l x (G, C).
  float4 va[4][4];
  float2 ab[4][4];  // rounded to FP32 at the load (the operand is FP32 before its TF32 split anyway)
  auto a_task = [&](int t, int h, int& acc, int& kk, int& pos0, int& comp) {
    if (NOPS == 1) {
      acc = t >> 3; kk = 4 * (t & 7); pos0 = acc * 32 + kk; comp = 0;
    } else {
      comp = t >> 3;
      const int par = (t >> 2) & 1, g4 = t & 3;
      acc = comp == 0 ? par : 1 - par;
      kk = 16 * comp + 4 * g4;
      pos0 = par * 32 + 16 * h + 4 * g4;
    }
  };
  auto load = [&](int st) {
    const int b = st / nhalf, h = st % nhalf;
    const float* unit0 = table + ((blockoff[m] + b) * int64_t(nquads) + q0) * UNIT;
    const bool qv = (q0 + lane) < nquads;
#pragma unroll
    for (int it = 0; it < 4; ++it) {
      int acc, kk, pos0, comp;
      a_task(warp + 4 * it, h, acc, kk, pos0, comp);
      const float* u = unit0 + int64_t(lane) * UNIT + (comp * TB_LB + pos0) * 4;
#pragma unroll
      for (int i = 0; i < 4; ++i)
        va[it][i] = qv ? __ldg(reinterpret_cast<const float4*>(u) + i) : make_float4(0.f, 0.f, 0.f, 0.f);
    }
    if (NOPS == 1) {
      const int j = lane;
#pragma unroll
      for (int i2 = 0; i2 < 4; ++i2) {
        const int t = warp + 4 * i2, acc = t >> 3, k4 = t & 7;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int l = tab_l(m, b, acc * 32 + 4 * k4 + i);
          const double2 a = (j < gs && l <= lmax) ? almT[(base + (l - m)) * B + b0 + j] : make_double2(0.0, 0.0);
          ab[i2][i] = make_float2(float(a.x), float(a.y));
        }
      }
    } else {
      const int j = lane & 15;
#pragma unroll
      for (int i2 = 0; i2 < 2; ++i2) {
        const int t = warp * 2 + (lane >> 4) + 8 * i2, acc = t >> 3, k4 = t & 7;
        const int comp = k4 >> 2, g4 = k4 & 3, par = comp == 0 ? acc : 1 - acc;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int l = tab_l(m, b, par * 32 + 16 * h + 4 * g4 + i);
          const bool v = j < gs && l <= lmax;
          const int64_t o = ((base + (l - m)) * B + b0 + j) * 2;
          const double2 G = v ? almT[o] : make_double2(0.0, 0.0), C = v ? almT[o + 1] : make_double2(0.0, 0.0);
          ab[2 * i2][i] = make_float2(float(G.x), float(G.y));
          ab[2 * i2 + 1][i] = make_float2(float(C.x), float(C.y));
        }
      }
    }
  };
  auto store = [&](int st) {
    const int h = st % nhalf;
#pragma unroll
    for (int it = 0; it < 4; ++it) {
      int acc, kk, pos0, comp;
      a_task(warp + 4 * it, h, acc, kk, pos0, comp);
      const int ks = kk >> 3, kc = (kk >> 2) & 1;
      const uint32_t oh = TabSmem::a(acc, ks, 0), ol = TabSmem::a(acc, ks, 1);
      // ring 4 lane + i of the tile -> A row 32 i + lane; rings outside [toff, toff + nrp) are zero
      const int rg0 = 4 * (q0 + lane);
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int rt = rg0 + i;
        const bool in = rt >= toff && rt < toff + nrp;
        float4 w;
        w.x = in ? (&va[it][0].x)[i] : 0.f;
        w.y = in ? (&va[it][1].x)[i] : 0.f;
        w.z = in ? (&va[it][2].x)[i] : 0.f;
        w.w = in ? (&va[it][3].x)[i] : 0.f;
        const uint32_t co = kcore_off(32 * i + lane, kc);
        st_split(c.smem, oh + co, ol + co, w);
      }
    }
    if (NOPS == 1) {
      const int j = lane;
      if (j < gs) {
#pragma unroll
        for (int i2 = 0; i2 < 4; ++i2) {
          const int t = warp + 4 * i2, acc = t >> 3, k4 = t & 7;
          const float4 re = make_float4(ab[i2][0].x, ab[i2][1].x, ab[i2][2].x, ab[i2][3].x);
          const float4 im = make_float4(ab[i2][0].y, ab[i2][1].y, ab[i2][2].y, ab[i2][3].y);
          const int ks = k4 >> 1, kc = k4 & 1;
          st_split(c.smem, TabSmem::b(acc, ks, 0) + kcore_off(j, kc), TabSmem::b(acc, ks, 1) + kcore_off(j, kc), re);
          st_split(c.smem, TabSmem::b(acc, ks, 0) + kcore_off(gs + j, kc),
                   TabSmem::b(acc, ks, 1) + kcore_off(gs + j, kc), im);
        }
      }
    } else {
      // F+ rows take X = -(G, C) (even spin) or Y = (C.im, -C.re, -G.im, G.re); F- rows the other one
      const int j = lane & 15;
      if (j < gs) {
#pragma unroll
        for (int i2 = 0; i2 < 2; ++i2) {
          const int t = warp * 2 + (lane >> 4) + 8 * i2, acc = t >> 3, k4 = t & 7;
          const int comp = k4 >> 2;
          const bool use_x = (comp == 0) != (spin_odd != 0);
          float4 pt[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const float2 G = ab[2 * i2][i], C = ab[2 * i2 + 1][i];
            float p0, p1, p2, p3;
            if (use_x) { p0 = -G.x; p1 = -G.y; p2 = -C.x; p3 = -C.y; }
            else { p0 = C.y; p1 = -C.x; p2 = -G.y; p3 = G.x; }
            (&pt[0].x)[i] = p0; (&pt[1].x)[i] = p1; (&pt[2].x)[i] = p2; (&pt[3].x)[i] = p3;
          }
          const int kk = 4 * k4, ks = kk >> 3, kc = (kk >> 2) & 1;
#pragma unroll
          for (int part = 0; part < 4; ++part) {
            const int row = part * gs + j;
            st_split(c.smem, TabSmem::b(acc, ks, 0) + kcore_off(row, kc), TabSmem::b(acc, ks, 1) + kcore_off(row, kc),
                     pt[part]);
          }
        }
      }
    }
  };
  uint32_t phase_bit = 0;
  bool ok = true;
  load(0);
  for (int st = 0; st < nst; ++st) {
    store(st);
    tab_issue_stage(c, idesc);
    if (st + 1 < nst) load(st + 1);
    ok = tab_finish_stage(c, n, st == 0, phase_bit, err_flag);
    if (!ok) break;
  }
  if (ok) {
    // epilogue: TMEM lane 32 w + q <-> ring 4 q + w of the tile
    const int rt = 4 * (q0 + lane) + warp;  // table ring
    const int i = rt - toff;                // ring pair of the plan
    const bool in = rt >= toff && i < nrp;
    const int R = 2 * nrp - 1;
    const int rs = R - 1 - i;
#pragma unroll 1
    for (int cb = 0; cb < n; cb += 16) {
      float s0[16], s1[16];
      tab_read_sum(c, 0, cb, s0);
      tab_read_sum(c, 1, cb, s1);
      if (!in) continue;
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const int col = cb + q;
        if (col >= ncols) break;
        const int part = col / gs, j = col % gs;
        const float nv = s0[q] + s1[q], sv = s0[q] - s1[q];
        float* pn = reinterpret_cast<float*>(phase + ((int64_t(i) * (mmax + 1) + m) * B + b0 + j) * NCOMP) + part;
        *pn = nv;
        if (rs != i) {
          float* ps_ = reinterpret_cast<float*>(phase + ((int64_t(rs) * (mmax + 1) + m) * B + b0 + j) * NCOMP) + part;
          *ps_ = sv;
        }
      }
    }
  }
  tab_end(c);
}

// ------------------------------------------------------------------ adjoint
// phase [R][mmax+1][B][NCOMP] complex64 of ring pairs [0, nrp) -> alm of map b at alm + b * out_stride
// ([NCOMP][nalm] complex128, times scale and lscale[comp][idx] when given), for the maps [b0, b0 + gs)
// of each group.  grid.x = map group + G * (entry of the (m, first block) work list)
template <int NOPS>
__global__ void __launch_bounds__(TB_THREADS, 2) tab_adj_kernel(const float* __restrict__ table,
                                                                 const int64_t* __restrict__ blockoff, int nquads,
                                                                 int toff, int nrp, int lmax, int mmax,
                                                                 const float2* __restrict__ phase,
                                                                 double2* __restrict__ alm, int B, int gsize,
                                                                 int ngroups, const int2* __restrict__ work,
                                                                 int64_t nalm, double scale, int spin_odd,
                                                                 int64_t out_stride,
                                                                 const double* __restrict__ lscale,
                                                                 int* __restrict__ err_flag) {
  constexpr int NCOMP = NOPS;
  constexpr int UNIT = NOPS * TB_LB * 4;
  constexpr int RSTAGE = NOPS == 1 ? 32 : 16;  // table rings per stage
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
  TabCta c = tab_begin(tab_smem_raw);
  const int nb = tab_nblocks(m, lmax);
  const int R = 2 * nrp - 1;
  const int rt_begin = toff & ~3, rt_end = toff + nrp;
  const int nstages = (rt_end - rt_begin + RSTAGE - 1) / RSTAGE;
  // Raw operands of one stage in registers (loaded while the previous stage's MMAs run).
  // A: NT (acc, blk, comp, quad) combinations, lane = position j, one float4 each (task t = warp + 4 i).
  // B: tasks (map j, quad qd) t = tid + 128 i: the north and south phases of 4 rings.
  constexpr int NQ = RSTAGE / 4;
  constexpr int NT = 2 * 4 * NOPS * NQ;  // (acc, blk, comp, quad) combinations
  constexpr int NA = NT / 4;
  constexpr int BT = NOPS == 1 ? 2 : 1;  // tasks per thread: NQ * gs <= 256 (spin 0) or 64 (spin s)
  float4 va[NA];
  float2 pn[BT][4][NCOMP], pv[BT][4][NCOMP];
  auto a_task = [&](int t, int& qd, int& comp, int& blk, int& acc) {
    qd = t % NQ;
    int r = t / NQ;
    comp = r % NOPS; r /= NOPS;
    blk = r % 4;
    acc = r / 4;
  };
  auto load = [&](int st) {
    const int rs0 = rt_begin + st * RSTAGE;  // first table ring of the stage (quad aligned)
#pragma unroll
    for (int i = 0; i < NA; ++i) {
      int qd, comp, blk, acc;
      a_task(warp + 4 * i, qd, comp, blk, acc);
      const int b = bb + blk;
      const int qg = rs0 / 4 + qd;
      float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
      if (b < nb && qg < nquads) {
        v = __ldg(reinterpret_cast<const float4*>(table + ((blockoff[m] + b) * int64_t(nquads) + qg) * UNIT +
                                                  (comp * TB_LB + acc * 32 + lane) * 4));
        // rings outside [toff, toff + nrp) contribute nothing
        const int r0 = 4 * qg;
        if (r0 < toff || r0 + 3 >= rt_end) {
          if (r0 + 0 < toff || r0 + 0 >= rt_end) v.x = 0.f;
          if (r0 + 1 < toff || r0 + 1 >= rt_end) v.y = 0.f;
          if (r0 + 2 < toff || r0 + 2 >= rt_end) v.z = 0.f;
          if (r0 + 3 < toff || r0 + 3 >= rt_end) v.w = 0.f;
        }
      }
      va[i] = v;
    }
#pragma unroll
    for (int bi = 0; bi < BT; ++bi) {
      const int t = tid + TB_THREADS * bi;
      const bool tv = t < NQ * gs;
      const int j = tv ? t % gs : 0, qd = tv ? t / gs : 0;
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int rt = rs0 + 4 * qd + i;
        const int ip = rt - toff;
        const bool in = tv && rt >= toff && ip < nrp;
        const int rsth = R - 1 - ip;
#pragma unroll
        for (int cc = 0; cc < NCOMP; ++cc) {
          pn[bi][i][cc] = in ? phase[((int64_t(ip) * (mmax + 1) + m) * B + b0 + j) * NCOMP + cc]
                             : make_float2(0.f, 0.f);
          pv[bi][i][cc] = (in && rsth != ip) ? phase[((int64_t(rsth) * (mmax + 1) + m) * B + b0 + j) * NCOMP + cc]
                                             : make_float2(0.f, 0.f);
        }
      }
    }
  };
  auto store = [&]() {
#pragma unroll
    for (int i = 0; i < NA; ++i) {
      int qd, comp, blk, acc;
      a_task(warp + 4 * i, qd, comp, blk, acc);
      const int kk = comp * 16 + 4 * qd;  // K index of the chunk (spin 0: comp = 0, qd < 8)
      const int ks = kk >> 3, kc = (kk >> 2) & 1;
      const int row = blk * 32 + lane;
      st_split(c.smem, TabSmem::a(acc, ks, 0) + kcore_off(row, kc), TabSmem::a(acc, ks, 1) + kcore_off(row, kc),
               va[i]);
    }
#pragma unroll
    for (int bi = 0; bi < BT; ++bi) {
      const int t = tid + TB_THREADS * bi;
      if (t >= NQ * gs) continue;
      const int j = t % gs, qd = t / gs;
      // ring sums (combo 0: N + S) and differences (combo 1: N - S) of 4 rings, per component
      float4 cre[2][NCOMP], cim[2][NCOMP];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int cc = 0; cc < NCOMP; ++cc) {
          const float2 nv = pn[bi][i][cc], sv = pv[bi][i][cc];
          (&cre[0][cc].x)[i] = nv.x + sv.x;
          (&cim[0][cc].x)[i] = nv.y + sv.y;
          (&cre[1][cc].x)[i] = nv.x - sv.x;
          (&cim[1][cc].x)[i] = nv.y - sv.y;
        }
      if (NOPS == 1) {
        const int kk = 4 * qd, ks = kk >> 3, kc = (kk >> 2) & 1;
#pragma unroll
        for (int acc = 0; acc < 2; ++acc) {
          st_split(c.smem, TabSmem::b(acc, ks, 0) + kcore_off(j, kc), TabSmem::b(acc, ks, 1) + kcore_off(j, kc),
                   cre[acc][0]);
          st_split(c.smem, TabSmem::b(acc, ks, 0) + kcore_off(gs + j, kc),
                   TabSmem::b(acc, ks, 1) + kcore_off(gs + j, kc), cim[acc][0]);
        }
      } else {
        // columns (G.re, G.im, C.re, C.im); combo k: Q = (cre[k][0], cim[k][0]), U = (cre[k][1], cim[k][1])
        // Xa(k) = (-Q.re, -Q.im, -U.re, -U.im), Ya(k) = (U.im, -U.re, -Q.im, Q.re)
        // even spin: F+ rows Xa(acc), F- rows Ya(1 - acc); odd spin: F+ rows Ya(acc), F- rows Xa(1 - acc)
#pragma unroll
        for (int acc = 0; acc < 2; ++acc) {
#pragma unroll
          for (int comp = 0; comp < 2; ++comp) {
            const int k = comp == 0 ? acc : 1 - acc;
            const bool use_x = (comp == 0) != (spin_odd != 0);
            const float4 qr = cre[k][0], qi = cim[k][0], ur = cre[k][NCOMP - 1], ui = cim[k][NCOMP - 1];
            float4 p[4];
            if (use_x) {
              p[0] = make_float4(-qr.x, -qr.y, -qr.z, -qr.w);
              p[1] = make_float4(-qi.x, -qi.y, -qi.z, -qi.w);
              p[2] = make_float4(-ur.x, -ur.y, -ur.z, -ur.w);
              p[3] = make_float4(-ui.x, -ui.y, -ui.z, -ui.w);
            } else {
              p[0] = ui;
              p[1] = make_float4(-ur.x, -ur.y, -ur.z, -ur.w);
              p[2] = make_float4(-qi.x, -qi.y, -qi.z, -qi.w);
              p[3] = qr;
            }
            const int kk = comp * 16 + 4 * qd, ks = kk >> 3, kc = (kk >> 2) & 1;
#pragma unroll
            for (int part = 0; part < 4; ++part) {
              const int row = part * gs + j;
              st_split(c.smem, TabSmem::b(acc, ks, 0) + kcore_off(row, kc),
                       TabSmem::b(acc, ks, 1) + kcore_off(row, kc), p[part]);
            }
          }
        }
      }
    }
  };
  uint32_t phase_bit = 0;
  bool ok = true;
  load(0);
  for (int st = 0; st < nstages; ++st) {
    store();
    tab_issue_stage(c, idesc);
    if (st + 1 < nstages) load(st + 1);
    ok = tab_finish_stage(c, n, st == 0, phase_bit, err_flag);
    if (!ok) break;
  }
  if (ok) {
    // epilogue: TMEM lane = A row = blk * 32 + j; accumulator acc is l = tab_l(m, bb + blk, acc * 32 + j)
    const int blk = warp, j = lane;
    const int b = bb + blk;
#pragma unroll 1
    for (int acc = 0; acc < 2; ++acc) {
      const int l = tab_l(m, b, acc * 32 + j);
      const bool in = b < nb && l <= lmax;
      const int64_t idx = alm_index(l, m, lmax);
#pragma unroll 1
      for (int cb = 0; cb < n; cb += 16) {
        float s[16];
        tab_read_sum(c, acc, cb, s);
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
  }
  tab_end(c);
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

// maps per group: as many as fit the 64 columns, spread evenly over the groups
static int tab_group_size(int B, int spin, int& ngroups) {
  const int cap = spin == 0 ? TB_NMAX / 2 : TB_NMAX / 4;
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
  int ngroups = 1;
  const int gsize = tab_group_size(B, spin, ngroups);
  const int ntiles = ((toff & 3) + P.Rh + TB_TILE - 1) / TB_TILE;
  const int nquads = tab_quads(Rh_table);
  const int64_t nblk = int64_t(ngroups) * ntiles * (P.mmax + 1);
  if (nblk > 0x7fffffff) return PS_ERR_UNSUPPORTED;
  const int smem = int(TabSmem::DYN);
  if (spin == 0) {
    if (set_smem_attr((const void*)tab_synth_kernel<1>, smem)) return PS_ERR_CUDA;
    tab_synth_kernel<1><<<unsigned(nblk), TB_THREADS, smem, st>>>(table, d_blockoff, nquads, toff, P.Rh, P.lmax,
                                                                  P.mmax, almT, phase, B, gsize, ngroups, ntiles, 0,
                                                                  err_flag);
  } else {
    if (set_smem_attr((const void*)tab_synth_kernel<2>, smem)) return PS_ERR_CUDA;
    tab_synth_kernel<2><<<unsigned(nblk), TB_THREADS, smem, st>>>(table, d_blockoff, nquads, toff, P.Rh, P.lmax,
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
  int ngroups = 1;
  const int gsize = tab_group_size(B, spin, ngroups);
  const int nquads = tab_quads(Rh_table);
  const int64_t nblk = int64_t(ngroups) * nwork;
  if (nblk > 0x7fffffff) return PS_ERR_UNSUPPORTED;
  const int smem = int(TabSmem::DYN);
  if (spin == 0) {
    if (set_smem_attr((const void*)tab_adj_kernel<1>, smem)) return PS_ERR_CUDA;
    tab_adj_kernel<1><<<unsigned(nblk), TB_THREADS, smem, st>>>(table, d_blockoff, nquads, toff, P.Rh, P.lmax,
                                                                P.mmax, phase, alm, B, gsize, ngroups, d_work,
                                                                P.nalm, scale, 0, out_stride, lscale, err_flag);
  } else {
    if (set_smem_attr((const void*)tab_adj_kernel<2>, smem)) return PS_ERR_CUDA;
    tab_adj_kernel<2><<<unsigned(nblk), TB_THREADS, smem, st>>>(table, d_blockoff, nquads, toff, P.Rh, P.lmax,
                                                                P.mmax, phase, alm, B, gsize, ngroups, d_work,
                                                                P.nalm, scale, spin & 1, out_stride, lscale,
                                                                err_flag);
  }
  PS_LAUNCH_CHECK();
  return PS_OK;
}

}  // namespace ps
