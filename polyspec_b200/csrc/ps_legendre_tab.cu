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
// 40 maps of spin 0 or 20 of spin s).
//
// Table layout.  For each order m the l range [m, lmax] is cut into blocks of
// 64 consecutive l.  Position j (0..31) of parity p of block b is
// l = m + 64b + 2j + p (zero beyond lmax); each block has two halves h, the
// positions 16h..16h+15 of both parities.  Ring pairs (north ring and its
// mirror, the equator last) are grouped in quads of 4.  One unit
// (m, b, h, quad q) is [ncomp][parity][16 positions][4 rings] FP32 (ncomp 1
// for spin 0, 2 for spin s: F+ then F-), and units are stored in the order
// (m, b, h, q), so that a synthesis stage (one half block of a 128-ring tile)
// is 32 runs of one unit.  A float4 of a unit is four consecutive rings at one
// l: a 16-byte row of a K-major core matrix of the adjoint's A operand (K =
// rings); the synthesis (K = l) transposes 4 x 4 blocks in registers.
//
// Both GEMMs split every FP32 operand into TF32 hi + lo and issue three MMAs
// per K step (hi.hi + hi.lo + lo.hi).  A stage is 16 K values per
// accumulator; operand tiles are double-buffered so that the MMAs of a stage
// run while the next stage is split.  The tensor core's FP32 accumulation
// truncates, so the accumulator D is restarted every two stages (32 K
// values) and added into a running sum S in TMEM (round-to-nearest FP32 adds
// by all 16 warps, the four warps of a TMEM lane quarter splitting the
// columns).  TMEM: D[2 buffers][2 accumulators][80] and S[2][80], so that the
// drain of one D overlaps the MMAs into the other.  One CTA of 16 warps per
// SM; one barrier per stage.
//
// Columns of D are (part, map) with the part index outermost: spin 0
// (re, im) of the complex value, spin s four real parts; map group g of up
// to 40 (spin 0) or 20 (spin s) maps.  N = the used columns rounded up to 16.
//
// Staging.  The table tiles (and, in the spin-s adjoint, the phase rows of
// the stage's rings) of up to four stages ahead are fetched by bulk copies
// (cp.async.bulk with mbarrier transaction counts); the a_lm (synthesis) and
// spin-0 phases (adjoint) of the next stage are loaded into registers.
//
// Synthesis (alm -> ring phases), CTA = (map group, ring tile of 128 ring
// pairs, m): M = ring pairs, K = l, two accumulators.  Spin 0: accumulator p
// sums the l of parity p; north ring = S0 + S1, south = S0 - S1.  Spin s:
// W = sum_even F+ u + sum_odd F- v and V = sum_odd F+ u + sum_even F- v (u, v
// the (Q, U) contributions of (G, C) through F+ and F-); north = W + V,
// south = W - V.  A stage of spin s is 8 positions of F+ (K 0..7) and of F-
// (K 8..15).
//
// Adjoint (ring phases -> alm), CTA = (map group, group of 4 l blocks, m):
// M = 128 l of one parity (32 positions of each of the 4 blocks), K = rings
// (16 per stage for spin 0; for spin s 8 rings as F+ rows and the same 8 as
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
// l of position j (0..31) of parity par of block b (may exceed lmax)
__host__ __device__ __forceinline__ int tab_l(int m, int b, int j, int par) { return m + TB_LB * b + 2 * j + par; }
// floats per unit (m, b, h, q): [ncomp][2 parities][16 positions][4 rings]
__host__ __device__ constexpr int tab_unit_floats(int ncomp) { return ncomp * 2 * 16 * 4; }
// stride of the units in the table (floats): 16 bytes of padding after each unit, so that a run of
// units lands in shared memory with the bank-spreading stride the transposing reads need, from one
// bulk copy (many small copies cap the copy engine at a fraction of HBM bandwidth)
__host__ __device__ constexpr int tab_unit_stride(int ncomp) { return tab_unit_floats(ncomp) + 4; }
// unit index of (global block gb = blockoff[m] + b, half h, quad q)
__host__ __device__ __forceinline__ int64_t tab_unit_index(int64_t gb, int h, int nquads, int q) {
  return (gb * 2 + h) * int64_t(nquads) + q;
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
// values go to a padded shared stage [2 halves][32 quads][unit + 4 floats] and then
// out to the table as two runs of 32 contiguous units.
template <int NOPS>
__global__ void __launch_bounds__(TB_THREADS) tab_gen_kernel(const RingInfo* __restrict__ rings,
                                                             const double* __restrict__ mnorm,
                                                             const SeedNorm* __restrict__ seednorm, int Rh, int lmax,
                                                             int spin, const int64_t* __restrict__ blockoff,
                                                             int nquads, float* __restrict__ table) {
  constexpr int UNIT = tab_unit_floats(NOPS);  // floats per unit
  constexpr int USTR = tab_unit_stride(NOPS);   // padded stride in the stage and the table
  extern __shared__ __align__(16) float tg_stage[];  // [2][32][USTR]
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
  for (int i = tid; i < 2 * 32 * USTR; i += TB_THREADS) tg_stage[i] = 0.f;  // the pads stay zero
  __syncthreads();
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
      // l = l0 + 2 jp + par: half jp >> 4, element ((comp * 2 + par) * 16 + (jp & 15)) * 4 of the unit
      const int jp = j >> 1, par = j & 1;
      const int pos = (jp >> 4) * 32 * USTR / 4 + par * 16 + (jp & 15);
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
        my[(32 + pos) * 4] = use ? float(0.5 * (f - gg)) : 0.f;
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
    // the 32 units of this tile are contiguous in the table, for each half
    for (int h = 0; h < 2; ++h) {
      // (padded units: the stage rows are the table's unit stride)
      float4* dst = reinterpret_cast<float4*>(table + tab_unit_index(blockoff[m] + b, h, nquads, tile * 32) * USTR);
      const float4* src = reinterpret_cast<const float4*>(tg_stage + h * 32 * USTR);
      for (int i = tid; i < 32 * USTR / 4; i += TB_THREADS) dst[i] = src[i];
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------------ MMA helpers
constexpr int TB_NMAX = 80;  // columns per accumulator (MMA N at most)

// K-major core matrices without swizzle: 8 rows x 16 bytes each, the two core matrices of an
// 8-wide K step 128 bytes apart, 8-row groups 256 bytes apart
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
__device__ __forceinline__ int round16(int x) { return (x + 15) & ~15; }

// Shared memory of one GEMM CTA.  Operand tiles, double-buffered by stage parity:
// A [buf][acc][ks][hi/lo] 4 KB each (128 rows x 8 K), B [buf][acc][ks][hi/lo] TB_NMAX x 32 B each;
// then NR staging buffers of RAW bytes for the bulk copies, then the pipeline's barriers, an abort
// flag and the TMEM slot (TabPipe).
template <uint32_t RAW, int NR_>
struct TabSmem {
  static constexpr int NR = NR_;
  static constexpr uint32_t RAW_BYTES = RAW;
  static constexpr uint32_t A_TILE = 128 * 32;
  static constexpr uint32_t B_TILE = TB_NMAX * 32;
  static constexpr uint32_t A_BUF = 8 * A_TILE;
  static constexpr uint32_t B_BUF = 8 * B_TILE;
  static constexpr uint32_t B_OFF = 2 * A_BUF;
  static constexpr uint32_t RAW_OFF = B_OFF + 2 * B_BUF;
  static constexpr uint32_t MISC_OFF = RAW_OFF + NR * RAW;
  static constexpr uint32_t DYN = MISC_OFF + 256 + 1024;  // + alignment of the base to 1 KB
  static constexpr uint32_t TMEM_COLS = 512;              // D[2][2][TB_NMAX], S[2][TB_NMAX]
  static_assert(RAW % 16 == 0 && NR <= 8, "staging buffers");
  __device__ static uint32_t a(int buf, int acc, int ks, int hl) {
    return uint32_t(buf) * A_BUF + uint32_t((acc * 2 + ks) * 2 + hl) * A_TILE;
  }
  __device__ static uint32_t b(int buf, int acc, int ks, int hl) {
    return B_OFF + uint32_t(buf) * B_BUF + uint32_t((acc * 2 + ks) * 2 + hl) * B_TILE;
  }
  __device__ static uint32_t raw(int i) { return RAW_OFF + uint32_t(i) * RAW; }
};

// TMEM columns: D[dbuf][acc] at (2 dbuf + acc) TB_NMAX, S[acc] at (4 + acc) TB_NMAX
__device__ __forceinline__ uint32_t tcol_d(int dbuf, int acc) { return uint32_t((2 * dbuf + acc) * TB_NMAX); }
__device__ __forceinline__ uint32_t tcol_s(int acc) { return uint32_t((4 + acc) * TB_NMAX); }

// CTA state shared by both GEMMs
struct TabCta {
  uint8_t* smem;
  uint32_t sbase;
  uint32_t tmem;
};

template <class S>
__device__ __forceinline__ void tab_end(const TabCta& c) {
  tc::fence_before_sync();
  __syncthreads();
  if ((threadIdx.x >> 5) == 0) tc::tmem_dealloc(c.tmem, S::TMEM_COLS);
}

// MMA issue.  Warp acc (0 or 1) issues the MMAs of accumulator acc, converged, one lane elected per
// instruction, from descriptors computed once per CTA (buffer 1: the buffer strides added to the
// start-address fields, which stay below 2^14 x 16 bytes); both warps commit to the stage's barrier
// (arrival count 2).  A single diverged lane that rebuilt the descriptors between MMAs fed the
// tensor core at about a third of this rate.
struct TabIssuer {
  uint64_t ah[2], al[2], bh[2], bl[2];  // buffer 0, K steps 0 and 1
  uint64_t da, db;                       // descriptor increments of buffer 1
  uint32_t d0;                           // TMEM address of D[0][acc]
};
template <class S>
__device__ __forceinline__ TabIssuer tab_issuer(const TabCta& c, int acc) {
  TabIssuer is;
#pragma unroll
  for (int ks = 0; ks < 2; ++ks) {
    is.ah[ks] = kdesc(c.sbase + S::a(0, acc, ks, 0));
    is.al[ks] = kdesc(c.sbase + S::a(0, acc, ks, 1));
    is.bh[ks] = kdesc(c.sbase + S::b(0, acc, ks, 0));
    is.bl[ks] = kdesc(c.sbase + S::b(0, acc, ks, 1));
  }
  is.da = uint64_t(S::A_BUF >> 4);
  is.db = uint64_t(S::B_BUF >> 4);
  is.d0 = c.tmem + tcol_d(0, acc);
  return is;
}
// one stage's MMAs of one accumulator: 2 K steps x (hi.hi + hi.lo + lo.hi) from operand buffer buf
// into D[dbuf]; restart: the first stage of a D period overwrites D.  Both operands K-major.  The
// tensor core's FP32 accumulator add truncates, with an error relative to the accumulator's
// magnitude: the small cross terms (hi.lo, lo.hi) go in first, while the accumulator is small, and
// the hi.hi products last, so that only those adds truncate at full magnitude.
__device__ __forceinline__ void tab_mma(const TabIssuer& is, int buf, int dbuf, bool restart, uint32_t idesc,
                                        uint32_t bar) {
  const uint64_t oa = buf ? is.da : 0, ob = buf ? is.db : 0;
  const uint32_t d = is.d0 + uint32_t(dbuf * 2 * TB_NMAX);
  tc::mma_tf32_elect(d, is.ah[0] + oa, is.bl[0] + ob, idesc, restart ? 0u : 1u);
  tc::mma_tf32_elect(d, is.ah[1] + oa, is.bl[1] + ob, idesc, 1u);
  tc::mma_tf32_elect(d, is.al[0] + oa, is.bh[0] + ob, idesc, 1u);
  tc::mma_tf32_elect(d, is.al[1] + oa, is.bh[1] + ob, idesc, 1u);
  tc::mma_tf32_elect(d, is.ah[0] + oa, is.bh[0] + ob, idesc, 1u);
  tc::mma_tf32_elect(d, is.ah[1] + oa, is.bh[1] + ob, idesc, 1u);
  tc::mma_commit_elect(bar);
}

// the S columns [cb, cb + 16) of accumulator acc of this thread's lane
__device__ __forceinline__ void tab_read_sum(const TabCta& c, int acc, int cb, float* v) {
  const uint32_t lane_addr = c.tmem + (uint32_t(((threadIdx.x >> 5) & 3) * 32) << 16);
  tc::tmem_ld16(lane_addr + tcol_s(acc) + uint32_t(cb), v);
  tc::tmem_ld_wait();
}

// ---- warp-specialised pipeline (synthesis).  Barriers at the start of the misc area, 8 bytes each:
// full[8] (staging buffer filled: bulk-copy transactions), raw_free[8] (staging buffer consumed:
// one arrival per producer warp), op_full[2] (operand buffer written: one per producer warp),
// mma_done[2] (the stage's MMAs complete: one commit per MMA warp), d_ready[2] (a D period's MMAs
// complete), d_free[2] (D drained into S: one arrival per drain warp); then an abort flag and the
// TMEM slot.
constexpr int WS_MMA_WARPS = 2;    // warps 0, 1: MMA issue, accumulator = warp
constexpr int WS_COPY_WARP = 2;    // bulk copies
constexpr int WS_PROD0 = 4;        // warps 4 .. 11: operand producers
constexpr int WS_NPROD = 8;
constexpr int WS_DRAIN0 = 12;      // warps 12 .. 15: drain, TMEM lane quarter = warp & 3
struct TabPipe {
  uint32_t full, raw_free, op_full, mma_done, d_ready, d_free;  // + 8 * index
  volatile int* abort;
};
template <class S>
__device__ __forceinline__ TabCta tab_begin_ws(uint8_t* smem_raw, TabPipe& pp) {
  TabCta c;
  c.smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  c.sbase = tc::smem_u32(c.smem);
  const uint32_t misc = c.sbase + S::MISC_OFF;
  pp.full = misc; pp.raw_free = misc + 64; pp.op_full = misc + 128; pp.mma_done = misc + 144;
  pp.d_ready = misc + 160; pp.d_free = misc + 176;
  pp.abort = reinterpret_cast<volatile int*>(c.smem + S::MISC_OFF + 192);
  uint32_t* slot = reinterpret_cast<uint32_t*>(c.smem + S::MISC_OFF + 224);
  if ((threadIdx.x >> 5) == 0) {
    tc::tmem_alloc(tc::smem_u32(slot), S::TMEM_COLS);
    tc::tmem_relinquish();
  }
  if (threadIdx.x == 0) {
    for (int i = 0; i < S::NR; ++i) {
      tc::mbar_init(pp.full + 8u * uint32_t(i), 1);
      tc::mbar_init(pp.raw_free + 8u * uint32_t(i), WS_NPROD);
    }
    for (int i = 0; i < 2; ++i) {
      tc::mbar_init(pp.op_full + 8u * uint32_t(i), WS_NPROD);
      tc::mbar_init(pp.mma_done + 8u * uint32_t(i), WS_MMA_WARPS);
      tc::mbar_init(pp.d_ready + 8u * uint32_t(i), WS_MMA_WARPS);
      tc::mbar_init(pp.d_free + 8u * uint32_t(i), 4);
    }
    *pp.abort = 0;
    tc::fence_mbar_init();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  c.tmem = *slot;
  return c;
}
// bounded wait of one warp (lane 0 polls, the result is shared): false when the limit is reached
// or another warp has aborted; the first to give up raises the abort flag and the error flag
__device__ __forceinline__ bool ws_wait(const TabPipe& pp, uint32_t mbar, uint32_t parity, int* err_flag) {
  int ok = 1;
  if ((threadIdx.x & 31) == 0) {
    ok = 0;
    for (uint32_t i = 0; i < TB_WAIT_LIMIT; ++i) {
      if (tc::mbar_try_wait(mbar, parity)) { ok = 1; break; }
      if ((i & 63) == 63 && *pp.abort) break;
    }
    if (!ok && atomicExch(const_cast<int*>(pp.abort), 1) == 0) atomicExch(err_flag, 1);
  }
  return __shfl_sync(0xffffffffu, ok, 0) != 0;
}
__device__ __forceinline__ void ws_arrive(uint32_t mbar) {
  __syncwarp();
  if ((threadIdx.x & 31) == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(mbar) : "memory");
}

// ------------------------------------------------------------------ synthesis
// staging of the synthesis: one half block (32 units) of a 128-ring tile per buffer, each unit at a
// padded stride (unit + 16 bytes) so that lanes reading different units hit different banks; a
// spin-s half block feeds two stages (8 positions each)
template <int NOPS>
struct SynthCfg {
  static constexpr int UNIT = tab_unit_floats(NOPS);
  static constexpr int USTR = tab_unit_stride(NOPS);
  static constexpr uint32_t RAW = 32u * USTR * 4u;
  static constexpr int NR = NOPS == 1 ? 7 : 3;  // as many as shared memory holds
  static constexpr int SPT = NOPS == 1 ? 1 : 2;  // stages per staged half block
};

// almT [nalm][B][NOPS] complex128 -> phase [R][mmax+1][B][NOPS] complex64 of the ring pairs
// [0, nrp) (table rings toff + i; north row i, south row R - 1 - i, R = 2 nrp - 1).
// grid.x = map group + G * (ring tile + T * m).
template <int NOPS>
__global__ void __launch_bounds__(TM_THREADS, 1) tab_synth_kernel(const float* __restrict__ table,
                                                                   const int64_t* __restrict__ blockoff, int nquads,
                                                                   int toff, int nrp, int lmax, int mmax,
                                                                   const double2* __restrict__ almT,
                                                                   float2* __restrict__ phase, int B, int gsize,
                                                                   int ngroups, int ntiles, int spin_odd,
                                                                   int* __restrict__ err_flag) {
  using G = SynthCfg<NOPS>;
  using S = TabSmem<G::RAW, G::NR>;
  constexpr int NCOMP = NOPS;
  constexpr int SPT = G::SPT;
  constexpr int NR = G::NR;
  constexpr int BSL = NOPS == 1 ? 2 : 1;  // B task slots per producer thread (8 gs <= 320 or 160)
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
  TabPipe pp;
  TabCta c = tab_begin_ws<S>(tab_smem_raw, pp);
  const int q0 = toff / 4 + tile * 32;  // first table quad of the tile
  const int nvq = max(0, min(32, nquads - q0));
  const int nb = tab_nblocks(m, lmax);
  const int nraw = 2 * nb;  // staged half blocks
  const int nst = nraw * SPT;
  const int64_t base = alm_index(m, m, lmax);
  const int64_t gb0 = blockoff[m];
  bool ok = true;
  int mma_issued = 0, raw_issued = 0;  // this warp's issued stages / half blocks (MMA and copy warps)

  if (warp < WS_MMA_WARPS) {
    // ---- MMA issue: stage s from operand buffer s & 1 into D[(s >> 1) & 1] (D period = 2 stages)
    const TabIssuer is = tab_issuer<S>(c, warp);
    for (int s = 0; s < nst && ok; ++s) {
      const int p = s >> 1;
      ok = ws_wait(pp, pp.op_full + 8u * uint32_t(s & 1), uint32_t(p & 1), err_flag);
      if (ok && (s & 1) == 0 && p >= 2) ok = ws_wait(pp, pp.d_free + 8u * uint32_t(p & 1), uint32_t((p >> 1) - 1) & 1u, err_flag);
      if (!ok) break;
      tc::fence_after_sync();
      tab_mma(is, s & 1, p & 1, (s & 1) == 0, idesc, pp.mma_done + 8u * uint32_t(s & 1));
      if (s & 1) tc::mma_commit_elect(pp.d_ready + 8u * uint32_t(p & 1));
      mma_issued = s + 1;
    }
  } else if (warp == WS_COPY_WARP) {
    // ---- bulk copies: half block r (block r >> 1, half r & 1) of the tile into staging buffer r % NR,
    // its nvq padded units in one copy
    for (int r = 0; r < nraw; ++r) {
      if (r >= NR) {
        ok = ws_wait(pp, pp.raw_free + 8u * uint32_t(r % NR), uint32_t((r / NR) - 1) & 1u, err_flag);
        if (!ok) break;
      }
      const uint32_t bar = pp.full + 8u * uint32_t(r % NR);
      if (lane == 0) {
        tc::mbar_arrive_expect_tx(bar, uint32_t(nvq) * G::USTR * 4u);
        if (nvq > 0)
          tc::bulk_g2s(c.sbase + S::raw(r % NR), table + tab_unit_index(gb0 + (r >> 1), r & 1, nquads, q0) * G::USTR,
                       uint32_t(nvq) * G::USTR * 4u, bar);
      }
      __syncwarp();
      raw_issued = r + 1;
    }
  } else if (warp >= WS_PROD0 && warp < WS_PROD0 + WS_NPROD) {
    // ---- operand producers (256 threads, pt = 0..255)
    const int pt = tid - 32 * WS_PROD0;
    // A: task pt (quad q = pt & 31, r = pt >> 5) loads 4 positions x 4 rings of quad q and stores them
    // transposed: ring 4 q + i of the tile is A row 32 i + q (the 16-byte stores of eight consecutive
    // lanes fall into eight different bank groups), K = 4 consecutive positions.
    // spin 0: (parity p, group g) = (r >> 2, r & 3), positions 4 g + i -> A(acc p, ks g >> 1, kc g & 1);
    // spin s (stage half qq): (comp cc, parity p, group g) = (r >> 2, (r >> 1) & 1, r & 1) at positions
    // 8 qq + 4 g + i -> A(acc = p for F+, 1 - p for F-; ks cc, kc g)
    int a_src;
    uint32_t a_dst;
    {
      const int q = pt & 31, r = (pt >> 5) & 7;
      int p, g, acc, ks, cc;
      if (NOPS == 1) {
        cc = 0; p = r >> 2; g = r & 3; acc = p; ks = g >> 1;
      } else {
        cc = r >> 2; p = (r >> 1) & 1; g = r & 1; acc = cc == 0 ? p : 1 - p; ks = cc;
      }
      a_src = q * G::USTR + ((cc * 2 + p) * 16 + 4 * g) * 4;  // spin s: + 32 qq
      a_dst = uint32_t(((acc * 2 + ks) * 2) * S::A_TILE) + kcore_off(q, g & 1);  // row 32 i + q: + 1024 i
    }
    // B: tasks t = pt + 256 k < 8 gs (map j = t % gs, (acc, k4) = t / gs), 4 K values of 2 (spin 0) or
    // 4 (spin s) rows.  K index 4 k4 + i of acc: spin 0 position 16 h + 4 k4 + i of parity acc;
    // spin s comp cc = k4 >> 1 at position 16 h + 8 qq + 4 (k4 & 1) + i, parity acc (F+) or 1 - acc (F-)
    bool b_v[BSL];
    int b_j[BSL], b_acc[BSL], b_k4[BSL], b_lofs[BSL];
#pragma unroll
    for (int k = 0; k < BSL; ++k) {
      const int t = pt + 256 * k;
      b_v[k] = t < 8 * gs;
      b_j[k] = b_v[k] ? t % gs : 0;
      const int ak = b_v[k] ? t / gs : 0;
      b_acc[k] = ak >> 2; b_k4[k] = ak & 3;
      const int cc = NOPS == 1 ? 0 : b_k4[k] >> 1;
      b_lofs[k] = NOPS == 1 ? 8 * b_k4[k] + b_acc[k] : 8 * (b_k4[k] & 1) + (cc == 0 ? b_acc[k] : 1 - b_acc[k]);
    }
    // the next stage's a_lm, loaded as FP64 and converted only when they are split (a conversion next
    // to the load would wait for it and prefetch nothing)
    double2 ab[BSL][NCOMP][4];
    auto load_alm = [&](int s) {
      const int r = s / SPT, qq = s % SPT, b = r >> 1, h = r & 1;
#pragma unroll
      for (int k = 0; k < BSL; ++k) {
        const int l0 = m + TB_LB * b + 32 * h + 16 * qq + b_lofs[k];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int l = l0 + 2 * i;
          const bool v = b_v[k] && l <= lmax;
          const int64_t o = ((base + (l - m)) * B + b0 + b_j[k]) * NCOMP;
#pragma unroll
          for (int cc = 0; cc < NCOMP; ++cc) {
            ab[k][cc][i] = v ? almT[o + cc] : make_double2(0.0, 0.0);
          }
        }
      }
    };
    load_alm(0);
    for (int s = 0; s < nst; ++s) {
      const int r = s / SPT, qq = s % SPT, buf = s & 1;
      if (qq == 0) ok = ws_wait(pp, pp.full + 8u * uint32_t(r % NR), uint32_t(r / NR) & 1u, err_flag);
      if (ok && s >= 2) ok = ws_wait(pp, pp.mma_done + 8u * uint32_t(buf), uint32_t((s - 2) >> 1) & 1u, err_flag);
      if (!ok) break;
      {  // A
        const float* u = reinterpret_cast<const float*>(c.smem + S::raw(r % NR)) + a_src + 32 * qq;
        float4 v[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) v[i] = reinterpret_cast<const float4*>(u)[i];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          // ring i of the quad: its values at the 4 positions
          const float4 w = make_float4((&v[0].x)[i], (&v[1].x)[i], (&v[2].x)[i], (&v[3].x)[i]);
          const uint32_t d = S::a(buf, 0, 0, 0) + a_dst + uint32_t(i) * kcore_off(32, 0);
          st_split(c.smem, d, d + S::A_TILE, w);
        }
      }
#pragma unroll
      for (int k = 0; k < BSL; ++k) {  // B
        if (!b_v[k]) continue;
        const int ks = b_k4[k] >> 1, kc = b_k4[k] & 1, j = b_j[k];
        const uint32_t bh = S::b(buf, b_acc[k], ks, 0), bl = S::b(buf, b_acc[k], ks, 1);
        if (NOPS == 1) {
          const float4 re = make_float4(float(ab[k][0][0].x), float(ab[k][0][1].x), float(ab[k][0][2].x),
                                        float(ab[k][0][3].x));
          const float4 im = make_float4(float(ab[k][0][0].y), float(ab[k][0][1].y), float(ab[k][0][2].y),
                                        float(ab[k][0][3].y));
          st_split(c.smem, bh + kcore_off(j, kc), bl + kcore_off(j, kc), re);
          st_split(c.smem, bh + kcore_off(gs + j, kc), bl + kcore_off(gs + j, kc), im);
        } else {
          // F+ rows take X = -(G, C) (even spin) or Y = (C.im, -C.re, -G.im, G.re); F- rows the other one
          const bool use_x = ((b_k4[k] >> 1) == 0) != (spin_odd != 0);
          float4 pt4[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const float2 Gv = make_float2(float(ab[k][0][i].x), float(ab[k][0][i].y));
            const float2 Cv = make_float2(float(ab[k][NCOMP - 1][i].x), float(ab[k][NCOMP - 1][i].y));
            float p0, p1, p2, p3;
            if (use_x) { p0 = -Gv.x; p1 = -Gv.y; p2 = -Cv.x; p3 = -Cv.y; }
            else { p0 = Cv.y; p1 = -Cv.x; p2 = -Gv.y; p3 = Gv.x; }
            (&pt4[0].x)[i] = p0; (&pt4[1].x)[i] = p1; (&pt4[2].x)[i] = p2; (&pt4[3].x)[i] = p3;
          }
#pragma unroll
          for (int part = 0; part < 4; ++part) {
            const int row = part * gs + j;
            st_split(c.smem, bh + kcore_off(row, kc), bl + kcore_off(row, kc), pt4[part]);
          }
        }
      }
      tc::fence_proxy_async();  // the operand stores, visible to the tensor core
      ws_arrive(pp.op_full + 8u * uint32_t(buf));
      if (qq == SPT - 1) ws_arrive(pp.raw_free + 8u * uint32_t(r % NR));  // half block r has been read
      if (s + 1 < nst) load_alm(s + 1);
    }
  } else if (warp >= WS_DRAIN0) {
    // ---- drain: S += D of each D period (first period: S = D), this warp's TMEM lane quarter,
    // all columns, two 16-column units per wait
    const uint32_t lane_addr = c.tmem + (uint32_t((warp & 3) * 32) << 16);
    const int nu = n >> 3;  // units u = (chunk u >> 1, accumulator u & 1)
    const int npairs = nst >> 1;
    for (int p = 0; p < npairs; ++p) {
      ok = ws_wait(pp, pp.d_ready + 8u * uint32_t(p & 1), uint32_t(p >> 1) & 1u, err_flag);
      if (!ok) break;
      tc::fence_after_sync();
      const bool first = p == 0;
#pragma unroll 1
      for (int u = 0; u < nu; u += 2) {
        float d0[16], d1[16], s0[16], s1[16];
        const bool two = u + 1 < nu;
        const uint32_t dc0 = lane_addr + tcol_d(p & 1, u & 1) + uint32_t(16 * (u >> 1));
        const uint32_t sc0 = lane_addr + tcol_s(u & 1) + uint32_t(16 * (u >> 1));
        const uint32_t dc1 = lane_addr + tcol_d(p & 1, (u + 1) & 1) + uint32_t(16 * ((u + 1) >> 1));
        const uint32_t sc1 = lane_addr + tcol_s((u + 1) & 1) + uint32_t(16 * ((u + 1) >> 1));
        tc::tmem_ld16(dc0, d0);
        if (!first) tc::tmem_ld16(sc0, s0);
        if (two) {
          tc::tmem_ld16(dc1, d1);
          if (!first) tc::tmem_ld16(sc1, s1);
        }
        tc::tmem_ld_wait();
        if (!first) {
#pragma unroll
          for (int q = 0; q < 16; ++q) { d0[q] += s0[q]; d1[q] += s1[q]; }
        }
        tmem_st16(sc0, d0);
        if (two) tmem_st16(sc1, d1);
      }
      tmem_st_wait();
      tc::fence_before_sync();
      ws_arrive(pp.d_free + 8u * uint32_t(p & 1));
    }
  }
  // every role has finished (or given up)
  tc::fence_before_sync();
  const bool failed = __syncthreads_or(!ok) != 0;
  tc::fence_after_sync();
  if (!failed) {
    // epilogue.  TMEM lane tl = 32 lq + q <-> ring 4 q + lq of the tile (lq = warp & 3).  The sums go
    // through shared memory (free now: every MMA and copy has completed) as rows [north/south][lane]
    // [map][part], then every ring's row of gs maps is written with coalesced stores
    constexpr int RS = TB_NMAX + 1;  // row stride (floats): consecutive lanes in consecutive banks
    static_assert(2 * 128 * RS * 4 <= int(S::MISC_OFF), "epilogue rows exceed the free shared memory");
    float* rows = reinterpret_cast<float*>(c.smem);
    const int lq = warp & 3, cs = warp >> 2;
    const int tl = 32 * lq + lane;
#pragma unroll 1
    for (int cb = 16 * cs; cb < n; cb += 64) {
      float s0[16], s1[16];
      tab_read_sum(c, 0, cb, s0);
      tab_read_sum(c, 1, cb, s1);
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
  } else if (lane == 0 && warp < WS_MMA_WARPS && mma_issued > 0) {
    // the issued MMAs read this CTA's shared memory and write its TMEM: wait (bounded) for them
    const int sp = mma_issued - 1;
    tc::mbar_wait_bounded(pp.mma_done + 8u * uint32_t(sp & 1), uint32_t(sp >> 1) & 1u, TB_WAIT_LIMIT);
  } else if (lane == 0 && warp == WS_COPY_WARP) {
    // copies in flight land in this CTA's shared memory: wait (bounded) for the last NR
    for (int k = max(0, raw_issued - NR); k < raw_issued; ++k)
      tc::mbar_wait_bounded(pp.full + 8u * uint32_t(k % NR), uint32_t(k / NR) & 1u, TB_WAIT_LIMIT);
  }
  tab_end<S>(c);
}

// ------------------------------------------------------------------ adjoint
// staging of one adjoint stage: for each of the 4 blocks and both halves, the NQ units of the
// stage's rings, [block][half][quad][unit]; spin s: then the north and south phase rows of the
// stage's rings, [north/south][ring][PH_MAPS maps] complex64 pairs
template <int NOPS>
struct AdjCfg {
  static constexpr int UNIT = tab_unit_floats(NOPS);
  static constexpr int NQ = NOPS == 1 ? 4 : 2;  // quads per stage
  static constexpr int RSTAGE = 4 * NQ;         // rings per stage
  static constexpr int USTR = tab_unit_stride(NOPS);
  static constexpr uint32_t TAB_BYTES = 8u * NQ * USTR * 4u;
  static constexpr int PH_MAPS = TB_NMAX / 4;   // maps per group (spin s)
  static constexpr uint32_t PH_BYTES = NOPS == 2 ? 2u * RSTAGE * PH_MAPS * 16u : 0u;
  static constexpr uint32_t RAW = TAB_BYTES + PH_BYTES;
  static constexpr int NR = NOPS == 1 ? 7 : 5;  // as many as shared memory holds
};

// phase [R][mmax+1][B][NOPS] complex64 of ring pairs [0, nrp) -> alm of map b at alm + b * out_stride
// ([NOPS][nalm] complex128, times scale and lscale[comp][idx] when given), for the maps [b0, b0 + gs)
// of each group.  grid.x = map group + G * (entry of the (m, first block) work list)
template <int NOPS>
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
  using G = AdjCfg<NOPS>;
  using S = TabSmem<G::RAW, G::NR>;
  constexpr int NCOMP = NOPS;
  constexpr int NQ = G::NQ;
  constexpr int RSTAGE = G::RSTAGE;
  constexpr int NR = G::NR;
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
  TabPipe pp;
  TabCta c = tab_begin_ws<S>(tab_smem_raw, pp);
  const int nb = tab_nblocks(m, lmax);
  const int nblk = min(4, nb - bb);
  const int R = 2 * nrp - 1;
  const int rt_begin = toff & ~3, rt_end = toff + nrp;
  const int nst = (rt_end - rt_begin + RSTAGE - 1) / RSTAGE;
  const int npairs = (nst + 1) >> 1;  // D periods (the last may hold one stage)
  const int64_t gb0 = blockoff[m] + bb;
  bool ok = true;
  int mma_issued = 0, raw_issued = 0;  // this warp's issued stages (MMA and copy warps)

  if (warp < WS_MMA_WARPS) {
    // ---- MMA issue: stage st from operand buffer st & 1 into D[(st >> 1) & 1]
    const TabIssuer is = tab_issuer<S>(c, warp);
    for (int st = 0; st < nst; ++st) {
      const int p = st >> 1;
      ok = ws_wait(pp, pp.op_full + 8u * uint32_t(st & 1), uint32_t(p & 1), err_flag);
      if (ok && (st & 1) == 0 && p >= 2) ok = ws_wait(pp, pp.d_free + 8u * uint32_t(p & 1), uint32_t((p >> 1) - 1) & 1u, err_flag);
      if (!ok) break;
      tc::fence_after_sync();
      tab_mma(is, st & 1, p & 1, (st & 1) == 0, idesc, pp.mma_done + 8u * uint32_t(st & 1));
      if ((st & 1) || st == nst - 1) tc::mma_commit_elect(pp.d_ready + 8u * uint32_t(p & 1));
      mma_issued = st + 1;
    }
  } else if (warp == WS_COPY_WARP) {
    // ---- bulk copies of stage st into staging buffer st % NR: lane 2 blk + h the units of block blk,
    // half h; spin s: lane r < RSTAGE the north and south phase rows of ring r of the stage
    for (int st = 0; st < nst; ++st) {
      if (st >= NR) {
        ok = ws_wait(pp, pp.raw_free + 8u * uint32_t(st % NR), uint32_t((st / NR) - 1) & 1u, err_flag);
        if (!ok) break;
      }
      const int rs0 = rt_begin + st * RSTAGE;
      const int qs = rs0 / 4;
      const int nvq = max(0, min(NQ, nquads - qs));
      uint32_t tx = uint32_t(nblk * 2 * nvq) * G::USTR * 4u;
      const int ip = rs0 + lane - toff;
      const bool ph_n = NOPS == 2 && lane < RSTAGE && ip >= 0 && ip < nrp;
      const bool ph_s = ph_n && R - 1 - ip != ip;
      const uint32_t row_bytes = uint32_t(gs) * 16u;
      if (NOPS == 2)
        tx += uint32_t(__popc(__ballot_sync(0xffffffffu, ph_n)) + __popc(__ballot_sync(0xffffffffu, ph_s))) * row_bytes;
      const uint32_t bar = pp.full + 8u * uint32_t(st % NR);
      const uint32_t dst = c.sbase + S::raw(st % NR);
      if (lane == 0) tc::mbar_arrive_expect_tx(bar, tx);
      __syncwarp();  // the transaction count is expected before any copy lands
      if (lane < 8 && (lane >> 1) < nblk && nvq > 0)
        tc::bulk_g2s(dst + uint32_t(lane * NQ * G::USTR) * 4u,
                     table + tab_unit_index(gb0 + (lane >> 1), lane & 1, nquads, qs) * G::USTR,
                     uint32_t(nvq) * G::USTR * 4u, bar);
      if (NOPS == 2) {
        const uint32_t pd = dst + G::TAB_BYTES + uint32_t(lane) * G::PH_MAPS * 16u;
        if (ph_n) tc::bulk_g2s(pd, phase + ((int64_t(ip) * (mmax + 1) + m) * B + b0) * NCOMP, row_bytes, bar);
        if (ph_s)
          tc::bulk_g2s(pd + uint32_t(RSTAGE) * G::PH_MAPS * 16u,
                       phase + ((int64_t(R - 1 - ip) * (mmax + 1) + m) * B + b0) * NCOMP, row_bytes, bar);
      }
      raw_issued = st + 1;
    }
  } else if (warp >= WS_PROD0 && warp < WS_PROD0 + WS_NPROD) {
    // ---- operand producers (256 threads, pt = 0..255)
    const int pt = tid - 32 * WS_PROD0;
    // A: float4 t = pt + 256 i (i = 0..3) of the stage's 1024: unit u = t / (32 NOPS) = (block, half,
    // quad qd) of the staged runs, element (comp cc, parity p, position jj) -> A(acc p), row
    // 32 block + 16 half + jj, K chunk cc NQ + qd (four rings)
    uint32_t a_dst[4];
    int a_qd[4], a_src[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int t = pt + 256 * i;
      const int u = t / (32 * NOPS), w = t % (32 * NOPS);
      a_src[i] = u * G::USTR + 4 * w;  // padded unit u of the staged runs
      const int cc = w >> 5, p = (w >> 4) & 1, jj = w & 15;
      const int qd = u % NQ, bh = u / NQ, h = bh & 1, blk = bh >> 1;
      const int row = blk * 32 + 16 * h + jj, kq = cc * NQ + qd;
      a_qd[i] = qd;
      a_dst[i] = uint32_t(((p * 2 + (kq >> 1)) * 2) * S::A_TILE) + kcore_off(row, kq & 1);
    }
    // B.  spin 0: task pt < NQ gs (map j = pt % gs, quad qd = pt / gs), phases of its 4 rings loaded
    // into registers a stage ahead.  spin s: task pt (acc = (pt >> 1) & 1, comp cc = pt & 1, map
    // j = (pt >> 2) % gs, quad qd = (pt >> 2) / gs), NQ gs <= 40, phases read from the staged rows
    const int p_t = NOPS == 1 ? pt : pt >> 2;
    const bool p_v = p_t < NQ * gs;
    const int p_j = p_v ? p_t % gs : 0, p_qd = p_v ? p_t / gs : 0;
    float2 pn[4], pv[4];
    auto load_phase = [&](int st) {
      if (NOPS != 1) return;
      const int rs0 = rt_begin + st * RSTAGE;
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int ip = rs0 + 4 * p_qd + i - toff;
        const bool in = p_v && ip >= 0 && ip < nrp;
        const int rsth = R - 1 - ip;
        pn[i] = in ? phase[(int64_t(ip) * (mmax + 1) + m) * B + b0 + p_j] : make_float2(0.f, 0.f);
        pv[i] = (in && rsth != ip) ? phase[(int64_t(rsth) * (mmax + 1) + m) * B + b0 + p_j] : make_float2(0.f, 0.f);
      }
    };
    load_phase(0);
    for (int st = 0; st < nst; ++st) {
      const int buf = st & 1;
      ok = ws_wait(pp, pp.full + 8u * uint32_t(st % NR), uint32_t(st / NR) & 1u, err_flag);
      if (ok && st >= 2) ok = ws_wait(pp, pp.mma_done + 8u * uint32_t(buf), uint32_t((st - 2) >> 1) & 1u, err_flag);
      if (!ok) break;
      const int rs0 = rt_begin + st * RSTAGE;
      const int nvq = max(0, min(NQ, nquads - rs0 / 4));
      const float* raw = reinterpret_cast<const float*>(c.smem + S::raw(st % NR));
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        // quads beyond the table were not copied: their rings contribute nothing
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (a_qd[i] < nvq) v = *reinterpret_cast<const float4*>(raw + a_src[i]);
        const uint32_t d = S::a(buf, 0, 0, 0) + a_dst[i];
        st_split(c.smem, d, d + S::A_TILE, v);
      }
      if (p_v && NOPS == 1) {
        const int j = p_j, qd = p_qd;
        // ring sums (accumulator 0: N + S) and differences (accumulator 1: N - S) of 4 rings
        float4 cre[2], cim[2];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          (&cre[0].x)[i] = pn[i].x + pv[i].x;
          (&cim[0].x)[i] = pn[i].y + pv[i].y;
          (&cre[1].x)[i] = pn[i].x - pv[i].x;
          (&cim[1].x)[i] = pn[i].y - pv[i].y;
        }
        const int ks = qd >> 1, kc = qd & 1;
#pragma unroll
        for (int acc = 0; acc < 2; ++acc) {
          const uint32_t bh = S::b(buf, acc, ks, 0), bl = S::b(buf, acc, ks, 1);
          st_split(c.smem, bh + kcore_off(j, kc), bl + kcore_off(j, kc), cre[acc]);
          st_split(c.smem, bh + kcore_off(gs + j, kc), bl + kcore_off(gs + j, kc), cim[acc]);
        }
      } else if (p_v) {
        // columns (G.re, G.im, C.re, C.im); combo k (0: N + S, 1: N - S) of the rings' (Q, U):
        // Xa(k) = (-Q.re, -Q.im, -U.re, -U.im), Ya(k) = (U.im, -U.re, -Q.im, Q.re)
        // even spin: F+ rows Xa(acc), F- rows Ya(1 - acc); odd spin: F+ rows Ya(acc), F- rows Xa(1 - acc)
        const int j = p_j, qd = p_qd;
        const int acc = (pt >> 1) & 1, cc = pt & 1;
        const int k = cc == 0 ? acc : 1 - acc;
        const bool use_x = (cc == 0) != (spin_odd != 0);
        const float4* ph = reinterpret_cast<const float4*>(c.smem + S::raw(st % NR) + G::TAB_BYTES);
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
        const int kq = cc * NQ + qd, ks = kq >> 1, kc = kq & 1;
        const uint32_t bh = S::b(buf, acc, ks, 0), bl = S::b(buf, acc, ks, 1);
#pragma unroll
        for (int part = 0; part < 4; ++part) {
          const int row = part * gs + j;
          st_split(c.smem, bh + kcore_off(row, kc), bl + kcore_off(row, kc), p[part]);
        }
      }
      tc::fence_proxy_async();  // the operand stores, visible to the tensor core
      ws_arrive(pp.op_full + 8u * uint32_t(buf));
      ws_arrive(pp.raw_free + 8u * uint32_t(st % NR));  // the stage's staged units and phase rows are read
      if (st + 1 < nst) load_phase(st + 1);
    }
  } else if (warp >= WS_DRAIN0) {
    // ---- drain: S += D of each D period (first period: S = D), this warp's TMEM lane quarter,
    // all columns, two 16-column units per wait
    const uint32_t lane_addr = c.tmem + (uint32_t((warp & 3) * 32) << 16);
    const int nu = n >> 3;  // units u = (chunk u >> 1, accumulator u & 1)
    for (int p = 0; p < npairs; ++p) {
      ok = ws_wait(pp, pp.d_ready + 8u * uint32_t(p & 1), uint32_t(p >> 1) & 1u, err_flag);
      if (!ok) break;
      tc::fence_after_sync();
      const bool first = p == 0;
#pragma unroll 1
      for (int u = 0; u < nu; u += 2) {
        float d0[16], d1[16], s0[16], s1[16];
        const bool two = u + 1 < nu;
        const uint32_t dc0 = lane_addr + tcol_d(p & 1, u & 1) + uint32_t(16 * (u >> 1));
        const uint32_t sc0 = lane_addr + tcol_s(u & 1) + uint32_t(16 * (u >> 1));
        const uint32_t dc1 = lane_addr + tcol_d(p & 1, (u + 1) & 1) + uint32_t(16 * ((u + 1) >> 1));
        const uint32_t sc1 = lane_addr + tcol_s((u + 1) & 1) + uint32_t(16 * ((u + 1) >> 1));
        tc::tmem_ld16(dc0, d0);
        if (!first) tc::tmem_ld16(sc0, s0);
        if (two) {
          tc::tmem_ld16(dc1, d1);
          if (!first) tc::tmem_ld16(sc1, s1);
        }
        tc::tmem_ld_wait();
        if (!first) {
#pragma unroll
          for (int q = 0; q < 16; ++q) { d0[q] += s0[q]; d1[q] += s1[q]; }
        }
        tmem_st16(sc0, d0);
        if (two) tmem_st16(sc1, d1);
      }
      tmem_st_wait();
      tc::fence_before_sync();
      ws_arrive(pp.d_free + 8u * uint32_t(p & 1));
    }
  }
  // every role has finished (or given up)
  tc::fence_before_sync();
  const bool failed = __syncthreads_or(!ok) != 0;
  tc::fence_after_sync();
  if (!failed && nst > 0) {
    // epilogue: TMEM lane = A row = 32 blk + j (blk = warp & 3, j = position in the parity), accumulator
    // acc is l = m + 64 (bb + blk) + 2 j + acc; the four warps of a lane quarter take every fourth
    // column chunk
    const int blk = warp & 3, cs = warp >> 2;
#pragma unroll 1
    for (int acc = 0; acc < 2; ++acc) {
      const int l = tab_l(m, bb + blk, lane, acc);
      const bool in = blk < nblk && l <= lmax;
      const int64_t idx = alm_index(l, m, lmax);
#pragma unroll 1
      for (int cb = 16 * cs; cb < n; cb += 64) {
        float sm[16];
        tab_read_sum(c, acc, cb, sm);
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
          *dst = double(sm[q]) * f;
        }
      }
    }
  } else if (failed && lane == 0 && warp < WS_MMA_WARPS && mma_issued > 0) {
    // the issued MMAs read this CTA's shared memory and write its TMEM: wait (bounded) for them
    const int sp = mma_issued - 1;
    tc::mbar_wait_bounded(pp.mma_done + 8u * uint32_t(sp & 1), uint32_t(sp >> 1) & 1u, TB_WAIT_LIMIT);
  } else if (failed && lane == 0 && warp == WS_COPY_WARP) {
    // copies in flight land in this CTA's shared memory: wait (bounded) for the last NR
    for (int k = max(0, raw_issued - NR); k < raw_issued; ++k)
      tc::mbar_wait_bounded(pp.full + 8u * uint32_t(k % NR), uint32_t(k / NR) & 1u, TB_WAIT_LIMIT);
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
  // two half-block units per block and quad, each padded
  return size_t(tab_total_blocks(lmax, mmax)) * size_t(tab_quads(Rh)) * 2 * size_t(tab_unit_stride(spin == 0 ? 1 : 2)) *
         sizeof(float);
}

int launch_tab_gen(const Plan& P, int spin, const int64_t* d_blockoff, float* table, cudaStream_t st) {
  const int nquads = tab_quads(P.Rh);
  dim3 grid(nquads * 4 / TB_TILE, P.mmax + 1);
  if (spin == 0) {
    const int smem = 2 * 32 * tab_unit_stride(1) * sizeof(float);
    if (set_smem_attr((const void*)tab_gen_kernel<1>, smem)) return PS_ERR_CUDA;
    tab_gen_kernel<1><<<grid, TB_THREADS, smem, st>>>(P.d_rings, P.d_mnorm0, nullptr, P.Rh, P.lmax, 0, d_blockoff,
                                                      nquads, table);
  } else {
    if (!P.d_seed[spin]) return PS_ERR_INVALID;
    const int smem = 2 * 32 * tab_unit_stride(2) * sizeof(float);
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
int launch_tab3_synth(const Plan& P, const uint16_t* table, const int64_t* d_blockoff, int Rh_table, int toff,
                      const double2* almT, float2* phase, int B, int spin, int* err_flag, cudaStream_t st);
int launch_tab3_adj(const Plan& P, const uint16_t* table, const int64_t* d_blockoff, const int2* d_work, int nwork,
                    int Rh_table, int toff, const float2* phase, double2* alm, int B, int spin, double scale,
                    int64_t out_stride, const double* lscale, int* err_flag, cudaStream_t st);

int launch_tab_synth(const Plan& P, const float* table, const int64_t* d_blockoff, int Rh_table, int toff,
                     const double2* almT, float2* phase, int B, int spin, int* err_flag, cudaStream_t st, int fmt) {
  if (fmt == PS_TAB_BF16X3)
    return launch_tab3_synth(P, reinterpret_cast<const uint16_t*>(table), d_blockoff, Rh_table, toff, almT, phase, B,
                             spin, err_flag, st);
  const double flops = double(spin == 0 ? 4 : 16) * double(P.Rh) * double(P.nalm) * B;
  const double bytes = double(tab_bytes(Rh_table, P.lmax, P.mmax, spin)) * double(P.Rh) / double(Rh_table) +
                       double(B) * (spin == 0 ? 1 : 2) * (16.0 * P.nalm + 8.0 * P.R * (P.mmax + 1));
  StatScope sc(PS_K_LEG_SYNTH, flops, bytes, st);
  // TB_NMAX columns per accumulator: up to 40 maps of spin 0 or 20 of spin s per pass over the table
  int ngroups = 1;
  const int gsize = tab_group_size(B, spin, TB_NMAX, ngroups);
  const int ntiles = ((toff & 3) + P.Rh + TB_TILE - 1) / TB_TILE;
  const int nquads = tab_quads(Rh_table);
  const int64_t nblk = int64_t(ngroups) * ntiles * (P.mmax + 1);
  if (nblk > 0x7fffffff) return PS_ERR_UNSUPPORTED;
  if (spin == 0) {
    const int smem = int(TabSmem<SynthCfg<1>::RAW, SynthCfg<1>::NR>::DYN);
    if (set_smem_attr((const void*)tab_synth_kernel<1>, smem)) return PS_ERR_CUDA;
    tab_synth_kernel<1><<<unsigned(nblk), TM_THREADS, smem, st>>>(table, d_blockoff, nquads, toff, P.Rh, P.lmax,
                                                                  P.mmax, almT, phase, B, gsize, ngroups, ntiles, 0,
                                                                  err_flag);
  } else {
    const int smem = int(TabSmem<SynthCfg<2>::RAW, SynthCfg<2>::NR>::DYN);
    if (set_smem_attr((const void*)tab_synth_kernel<2>, smem)) return PS_ERR_CUDA;
    tab_synth_kernel<2><<<unsigned(nblk), TM_THREADS, smem, st>>>(table, d_blockoff, nquads, toff, P.Rh, P.lmax,
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
                   int64_t out_stride, const double* lscale, int* err_flag, cudaStream_t st, int fmt) {
  if (fmt == PS_TAB_BF16X3)
    return launch_tab3_adj(P, reinterpret_cast<const uint16_t*>(table), d_blockoff, d_work, nwork, Rh_table, toff,
                           phase, alm, B, spin, scale, out_stride, lscale, err_flag, st);
  const double flops = double(spin == 0 ? 4 : 16) * double(P.Rh) * double(P.nalm) * B;
  const double bytes = double(tab_bytes(Rh_table, P.lmax, P.mmax, spin)) * double(P.Rh) / double(Rh_table) +
                       double(B) * (spin == 0 ? 1 : 2) * (16.0 * P.nalm + 8.0 * P.R * (P.mmax + 1));
  StatScope sc(PS_K_LEG_ADJOINT, flops, bytes, st);
  // TB_NMAX columns per accumulator: up to 40 maps of spin 0 or 20 of spin s per pass over the table
  int ngroups = 1;
  const int gsize = tab_group_size(B, spin, TB_NMAX, ngroups);
  const int nquads = tab_quads(Rh_table);
  const int64_t nblk = int64_t(ngroups) * nwork;
  if (nblk > 0x7fffffff) return PS_ERR_UNSUPPORTED;
  // spin s phase rows are staged by bulk copies, which start on 16-byte boundaries
  if (spin != 0 && (reinterpret_cast<uintptr_t>(phase) & 15u)) return PS_ERR_INVALID;
  if (spin == 0) {
    const int smem = int(TabSmem<AdjCfg<1>::RAW, AdjCfg<1>::NR>::DYN);
    if (set_smem_attr((const void*)tab_adj_kernel<1>, smem)) return PS_ERR_CUDA;
    tab_adj_kernel<1><<<unsigned(nblk), TM_THREADS, smem, st>>>(table, d_blockoff, nquads, toff, P.Rh, P.lmax,
                                                                      P.mmax, phase, alm, B, gsize, ngroups, d_work,
                                                                      P.nalm, scale, 0, out_stride, lscale, err_flag);
  } else {
    const int smem = int(TabSmem<AdjCfg<2>::RAW, AdjCfg<2>::NR>::DYN);
    if (set_smem_attr((const void*)tab_adj_kernel<2>, smem)) return PS_ERR_CUDA;
    tab_adj_kernel<2><<<unsigned(nblk), TM_THREADS, smem, st>>>(table, d_blockoff, nquads, toff, P.Rh, P.lmax,
                                                                      P.mmax, phase, alm, B, gsize, ngroups, d_work,
                                                                      P.nalm, scale, spin & 1, out_stride, lscale,
                                                                      err_flag);
  }
  PS_LAUNCH_CHECK();
  return PS_OK;
}

}  // namespace ps
