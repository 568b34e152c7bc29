// Table-driven Legendre stages, BF16x3 table format (tcgen05 kind::f16, accumulators in TMEM).
//
// The same normalised Legendre values as the FP32 table (FP64 recurrence, rounded to FP32), each
// split into three BF16 planes hi + mid + lo (24 significant bits together) and stored already in
// the tensor core's operand layout, so that both GEMMs stream the table straight from HBM into the
// MMA operand buffers by bulk copies: no operand-producing warps touch the table.
//
// Core matrix: 8 table positions (l of one parity) x 8 consecutive rings, BF16, rings contiguous
// (16 bytes per position, 128 bytes).  Read K-major it is the adjoint's A (M = l, K = rings); read
// MN-major it is the synthesis's A (M = rings, K = l).  For the MN-major no-swizzle descriptor the
// leading byte offset is the stride between K-adjacent core matrices and the stride byte offset the
// stride between M-adjacent ones, as for K-major (checked against a host GEMM on B200 with two
// layouts of different strides).
//
// Units.  For each order m the l range [m, lmax] is cut into blocks of 64 l (position j = 0..31 of
// parity p is l = m + 64 b + 2 j + p, zero beyond lmax); rings (north ring pairs, the equator last)
// in slabs Q of 16.  Unit (global block gb, slab Q) =
//   [r8 2][pos8 4][comp NC][parity 2][plane 3][8 positions][8 rings]  BF16
// (r8: the 8-ring half of the slab, pos8: positions 8 pos8 .. 8 pos8 + 7, comp: F+ / F- for spin s),
// 6 KB for spin 0 and 12 KB for spin s, at unit index gb * nQ + Q.
//
// Synthesis stage (block b, 16 K values): spin 0 both halves' 8-position groups pos8 = 2h, 2h + 1 of
// parity acc; spin s the 8 positions pos8 of F+ (parity acc) then of F- (parity 1 - acc).  A tile =
// 8 slabs (128 rings, M-adjacent core matrices 3072 bytes apart); a staging buffer holds two stages.
// Adjoint stage: 16 K values (spin 0: the 16 rings of a slab; spin s: 8 rings as F+ then F-) of the 4
// blocks of the CTA (128 l of parity acc, M-adjacent core matrices 768 / 1536 bytes apart).
//
// Products per 16 K and accumulator: lo.hi, hi.lo, mid.mid, mid.hi, hi.mid, hi.hi (the terms of
// order 2^-16 and above; the small ones first while the accumulator is small), FP32 accumulation in
// TMEM with the D-period restart and round-to-nearest running sums of the TF32x3 kernels.
#include <algorithm>
#include <vector>

#include <cuda_bf16.h>

#include "ps_common.cuh"
#include "ps_stats.cuh"
#include "ps_tc.cuh"

namespace ps {
// the table geometry shared with the FP32 format (ps_legendre_tab.cu)
int64_t tab_total_blocks(int lmax, int mmax);

namespace t3 {

constexpr int LB = 64;          // l per block
constexpr int TILE = 128;       // rings per synthesis tile
constexpr int NMAX = 80;        // accumulator columns
constexpr int THREADS = 512;    // GEMM CTAs: 16 warps
constexpr int GEN_THREADS = 128;
constexpr uint32_t WAIT_LIMIT = 1u << 24;
constexpr int MMA_WARPS = 2, COPY_WARP = 2, PROD0 = 4, NPROD = 8, DRAIN0 = 12;

template <int NC>
struct U {
  static constexpr uint32_t PLANE = 128;
  static constexpr uint32_t PAR = 3 * PLANE;
  static constexpr uint32_t COMP = 2 * PAR;
  static constexpr uint32_t POS8 = NC * COMP;
  static constexpr uint32_t R8 = 4 * POS8;
  static constexpr uint32_t UNIT = 2 * R8;
};

__host__ __device__ __forceinline__ int nblocks(int m, int lmax) { return (lmax - m) / LB + 1; }
__host__ __device__ __forceinline__ int nslabs(int Rh) { return ((Rh + TILE - 1) / TILE) * TILE / 16; }

__device__ __forceinline__ uint16_t bf16_bits(float x) {
  const __nv_bfloat16 h = __float2bfloat16_rn(x);
  return *reinterpret_cast<const uint16_t*>(&h);
}
__device__ __forceinline__ float bf16_float(uint16_t b) { return __uint_as_float(uint32_t(b) << 16); }
// v = hi + mid + lo (each BF16; exact residuals in FP32)
__device__ __forceinline__ void split3(float v, uint16_t& hi, uint16_t& mid, uint16_t& lo) {
  hi = bf16_bits(v);
  const float r1 = v - bf16_float(hi);
  mid = bf16_bits(r1);
  lo = bf16_bits(r1 - bf16_float(mid));
}

// seeds, as the FP32 table generator
__device__ __forceinline__ void seed0(int m, double sth, double mnorm, double& v, int& k) {
  Scaled s = smul(spow(sth, m), snorm(mnorm));
  to_kscale(s, v, k);
  if (m & 1) v = -v;
}
__device__ __forceinline__ void seedS(int m, int s, const RingInfo& g, SeedNorm nrm, double& f, double& gg, int& k) {
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

// One CTA = 128 rings (8 slabs) of one order m; thread = ring.  Block by block the three planes of
// the 64 values go to a shared stage laid out as the block's 8 units, then out as one contiguous run.
template <int NC>
__global__ void __launch_bounds__(GEN_THREADS) gen_kernel(const RingInfo* __restrict__ rings,
                                                           const double* __restrict__ mnorm,
                                                           const SeedNorm* __restrict__ seednorm, int Rh, int lmax,
                                                           int spin, const int64_t* __restrict__ blockoff, int nQ,
                                                           uint16_t* __restrict__ table) {
  using u = U<NC>;
  extern __shared__ __align__(16) uint8_t t3_gen_stage[];  // [8 units]
  __shared__ double s_c0[LB], s_c1[LB], s_c2[LB];
  const int m = blockIdx.y, tile = blockIdx.x, tid = threadIdx.x;
  const int rp = tile * TILE + tid;
  const bool active = rp < Rh;
  const RingInfo g = rings[active ? rp : 0];
  const double x = g.z;
  const int lmin = NC == 1 ? m : max(m, spin);
  double f = 0.0, fp = 0.0, gg = 0.0, gp = 0.0, sf = 0.0, sg = 0.0;
  int k = 0;
  if (NC == 1) seed0(m, g.sth, mnorm[m], f, k);
  else seedS(m, spin, g, seednorm[m], sf, sg, k);
  if (!active) { f = 0.0; sf = 0.0; sg = 0.0; k = 0; }
  // this thread's ring inside the stage: unit tid >> 4, half (tid >> 3) & 1, ring tid & 7
  uint8_t* my = t3_gen_stage + (tid >> 4) * u::UNIT + ((tid >> 3) & 1) * u::R8 + (tid & 7) * 2;
  const int nb = nblocks(m, lmax);
  for (int b = 0; b < nb; ++b) {
    const int l0 = m + LB * b;
    if (tid < LB) {
      double c0 = 0.0, c1 = 0.0, c2 = 0.0;
      if (NC == 1) {  // lam_{l+1} = c0 x lam_l - c1 lam_{l-1}, l = l0 + tid
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
    for (int j = 0; j < LB; ++j) {
      const int l = l0 + j;
      const int jp = j >> 1, par = j & 1;  // position jp (0..31), parity
      uint8_t* e = my + (jp >> 3) * u::POS8 + par * u::PAR + (jp & 7) * 16;
      float v0 = 0.f, v1 = 0.f;
      if (NC == 1) {
        if (k == 0 && l <= lmax) v0 = float(f);
        const double nxt = s_c0[j] * x * f - s_c1[j] * fp;
        fp = f;
        f = nxt;
        if (k < 0 && fabs(f) > PS_FTHRESH) { f *= PS_FSMALL; fp *= PS_FSMALL; ++k; }
      } else {
        if (l == lmin) { f = sf; gg = sg; fp = 0.0; gp = 0.0; }
        if (k == 0 && l <= lmax) { v0 = float(0.5 * (f + gg)); v1 = float(0.5 * (f - gg)); }
        const double ax = s_c0[j] * x;
        const double fn = (ax + s_c1[j]) * f - s_c2[j] * fp;
        const double gn = (ax - s_c1[j]) * gg - s_c2[j] * gp;
        fp = f; f = fn; gp = gg; gg = gn;
        if (k < 0 && fmax(fabs(f), fabs(gg)) > PS_FTHRESH) {
          f *= PS_FSMALL; fp *= PS_FSMALL; gg *= PS_FSMALL; gp *= PS_FSMALL; ++k;
        }
      }
#pragma unroll
      for (int cc = 0; cc < NC; ++cc) {
        uint16_t h, md, lo;
        split3(cc == 0 ? v0 : v1, h, md, lo);
        uint8_t* ec = e + cc * u::COMP;
        *reinterpret_cast<uint16_t*>(ec) = h;
        *reinterpret_cast<uint16_t*>(ec + u::PLANE) = md;
        *reinterpret_cast<uint16_t*>(ec + 2 * u::PLANE) = lo;
      }
    }
    __syncthreads();
    // the tile's 8 units of this block are one contiguous run of the table
    const int nq = min(8, nQ - tile * 8);
    int4* dst = reinterpret_cast<int4*>(reinterpret_cast<uint8_t*>(table) +
                                        (int64_t(blockoff[m] + b) * nQ + tile * 8) * int64_t(u::UNIT));
    const int4* src = reinterpret_cast<const int4*>(t3_gen_stage);
    for (int i = tid; i < nq * int(u::UNIT / 16); i += GEN_THREADS) dst[i] = src[i];
    __syncthreads();
  }
}


// ------------------------------------------------------------------ GEMM pipeline
// K-major / MN-major no-swizzle descriptor with explicit strides (bytes)
__device__ __forceinline__ uint64_t desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= uint64_t((saddr & 0x3FFFFu) >> 4);
  d |= uint64_t(lbo >> 4) << 16;
  d |= uint64_t(sbo >> 4) << 32;
  d |= uint64_t(1) << 46;
  return d;
}
// byte offset of (row, k) in a K-major B tile [rows][16 K] of BF16: 8 x 8 core matrices, K halves
// 128 bytes apart, 8-row groups 256 bytes apart
__device__ __forceinline__ uint32_t bcore(int row, int kg) { return uint32_t(((row >> 3) * 2 + kg) * 128 + (row & 7) * 16); }
__device__ __forceinline__ int round16(int x) { return (x + 15) & ~15; }

// Shared memory: NR staging buffers of RAW bytes (A straight from the table), then NB B operand
// buffers [buf][acc][plane] of NMAX x 16 BF16 each (the producers run up to NB - 1 stages ahead of
// the tensor core), then barriers, abort flag, TMEM slot.
constexpr int NB = 4;
template <uint32_t RAW_, int NR_>
struct Smem {
  static constexpr uint32_t RAW = RAW_;
  static constexpr int NR = NR_;
  static constexpr uint32_t BT = NMAX * 32;             // one B tile
  static constexpr uint32_t B_OFF = NR * RAW;
  static constexpr uint32_t MISC_OFF = B_OFF + NB * 6 * BT;
  static constexpr uint32_t DYN = MISC_OFF + 256 + 1024;
  static constexpr uint32_t TMEM_COLS = 512;             // D[2][2][NMAX], S[2][NMAX]
  static_assert(NR <= 8 && RAW % 128 == 0, "staging");
  __device__ static uint32_t raw(int i) { return uint32_t(i) * RAW; }
  __device__ static uint32_t b(int buf, int acc, int plane) { return B_OFF + uint32_t((buf * 2 + acc) * 3 + plane) * BT; }
};
__device__ __forceinline__ uint32_t tcol_d(int dbuf, int acc) { return uint32_t((2 * dbuf + acc) * NMAX); }
__device__ __forceinline__ uint32_t tcol_s(int acc) { return uint32_t((4 + acc) * NMAX); }

struct Pipe {
  uint32_t full, raw_free, op_full, mma_done, d_ready, d_free;
  volatile int* abort;
};
struct Cta {
  uint8_t* smem;
  uint32_t sbase, tmem;
};
// raw_free arrivals: one commit per MMA warp (the MMAs read A from the staging buffer)
template <class S>
__device__ __forceinline__ Cta begin(uint8_t* smem_raw, Pipe& pp) {
  Cta c;
  c.smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  c.sbase = tc::smem_u32(c.smem);
  const uint32_t misc = c.sbase + S::MISC_OFF;
  pp.full = misc; pp.raw_free = misc + 64; pp.op_full = misc + 128; pp.mma_done = misc + 128 + 8 * NB;
  pp.d_ready = misc + 128 + 16 * NB; pp.d_free = misc + 144 + 16 * NB;
  pp.abort = reinterpret_cast<volatile int*>(c.smem + S::MISC_OFF + 160 + 16 * NB);
  uint32_t* slot = reinterpret_cast<uint32_t*>(c.smem + S::MISC_OFF + 168 + 16 * NB);
  if ((threadIdx.x >> 5) == 0) {
    tc::tmem_alloc(tc::smem_u32(slot), S::TMEM_COLS);
    tc::tmem_relinquish();
  }
  if (threadIdx.x == 0) {
    for (int i = 0; i < S::NR; ++i) {
      tc::mbar_init(pp.full + 8u * uint32_t(i), 1);
      tc::mbar_init(pp.raw_free + 8u * uint32_t(i), MMA_WARPS);
    }
    for (int i = 0; i < NB; ++i) {
      tc::mbar_init(pp.op_full + 8u * uint32_t(i), NPROD);
      tc::mbar_init(pp.mma_done + 8u * uint32_t(i), MMA_WARPS);
    }
    for (int i = 0; i < 2; ++i) {
      tc::mbar_init(pp.d_ready + 8u * uint32_t(i), MMA_WARPS);
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
// bounded wait of one warp (lane 0 polls, the result is shared); the first to give up raises the
// CTA's abort flag and the plan's error flag
__device__ __forceinline__ bool wait(const Pipe& pp, uint32_t mbar, uint32_t parity, int* err_flag) {
  int ok = 1;
  if ((threadIdx.x & 31) == 0) {
    ok = 0;
    for (uint32_t i = 0; i < WAIT_LIMIT; ++i) {
      if (tc::mbar_try_wait(mbar, parity)) { ok = 1; break; }
      if ((i & 63) == 63 && *pp.abort) break;
    }
    if (!ok && atomicExch(const_cast<int*>(pp.abort), 1) == 0) atomicExch(err_flag, 1);
  }
  return __shfl_sync(0xffffffffu, ok, 0) != 0;
}
__device__ __forceinline__ void arrive(uint32_t mbar) {
  __syncwarp();
  if ((threadIdx.x & 31) == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(mbar) : "memory");
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

// six BF16 products of one stage and accumulator: A planes a0 + 128 k, B planes b0 + BT k
// (k = 0 hi, 1 mid, 2 lo); restart: the first product overwrites D
__device__ __forceinline__ void mma6(uint32_t d, uint32_t a0, uint32_t alb, uint32_t asb, uint32_t b0, uint32_t bt,
                                     uint32_t idesc, bool restart) {
  const uint64_t ah = desc(a0, alb, asb), am = desc(a0 + 128u, alb, asb), al = desc(a0 + 256u, alb, asb);
  const uint64_t bh = desc(b0, 128u, 256u), bm = desc(b0 + bt, 128u, 256u), bl = desc(b0 + 2u * bt, 128u, 256u);
  tc::mma_f16_elect(d, al, bh, idesc, restart ? 0u : 1u);
  tc::mma_f16_elect(d, ah, bl, idesc, 1u);
  tc::mma_f16_elect(d, am, bm, idesc, 1u);
  tc::mma_f16_elect(d, am, bh, idesc, 1u);
  tc::mma_f16_elect(d, ah, bm, idesc, 1u);
  tc::mma_f16_elect(d, ah, bh, idesc, 1u);
}

// write 8 values (K group kg of `row`) of a B operand as three planes
__device__ __forceinline__ void st_b8(uint8_t* smem, uint32_t plane0, uint32_t bt, int row, int kg, const float* v) {
  uint32_t w[3][4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    uint16_t h0, m0, l0, h1, m1, l1;
    split3(v[2 * i], h0, m0, l0);
    split3(v[2 * i + 1], h1, m1, l1);
    w[0][i] = uint32_t(h0) | (uint32_t(h1) << 16);
    w[1][i] = uint32_t(m0) | (uint32_t(m1) << 16);
    w[2][i] = uint32_t(l0) | (uint32_t(l1) << 16);
  }
  const uint32_t off = bcore(row, kg);
#pragma unroll
  for (int pl = 0; pl < 3; ++pl)
    *reinterpret_cast<uint4*>(smem + plane0 + pl * bt + off) = make_uint4(w[pl][0], w[pl][1], w[pl][2], w[pl][3]);
}

// drain of D period p into the running sums S (first period: S = D), this warp's lane quarter
__device__ __forceinline__ void drain(uint32_t tmem, int warp, int n, int p) {
  const uint32_t lane_addr = tmem + (uint32_t((warp & 3) * 32) << 16);
  const int nu = n >> 3;
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
}
__device__ __forceinline__ void read_sum(uint32_t tmem, int acc, int cb, float* v) {
  const uint32_t lane_addr = tmem + (uint32_t(((threadIdx.x >> 5) & 3) * 32) << 16);
  tc::tmem_ld16(lane_addr + tcol_s(acc) + uint32_t(cb), v);
  tc::tmem_ld_wait();
}


// ------------------------------------------------------------------ synthesis
// staging buffer = two stages: spin 0 the tile's 8 units of one block; spin s 16 pieces
// (slab, ring half) of 3 KB = the two position groups of the buffer
constexpr uint32_t SYN_RAW = 16u * 3072u;
constexpr int SYN_NR = 3;

// almT [nalm][B][NC] complex128 -> phase [R][mmax+1][B][NC] complex64 of the ring pairs [0, nrp) (table
// rings toff + i).  grid.x = map group + G * (ring tile + T * m).
template <int NC>
__global__ void __launch_bounds__(THREADS, 1) synth_kernel(const uint16_t* __restrict__ table,
                                                           const int64_t* __restrict__ blockoff, int nQ, int toff,
                                                           int nrp, int lmax, int mmax,
                                                           const double2* __restrict__ almT,
                                                           float2* __restrict__ phase, int B, int gsize, int ngroups,
                                                           int ntiles, int spin_odd, int* __restrict__ err_flag) {
  using u = U<NC>;
  using S = Smem<SYN_RAW, SYN_NR>;
  constexpr int NR = S::NR;
  extern __shared__ uint8_t t3_smem_raw[];
  int bid = blockIdx.x;
  const int grp = bid % ngroups; bid /= ngroups;
  const int tile = bid % ntiles;
  const int m = bid / ntiles;
  const int b0 = grp * gsize;
  const int gs = min(gsize, B - b0);
  const int ncols = 2 * NC * gs;
  const int n = round16(ncols);
  const uint32_t idesc = tc::idesc_bf16(128, n, 1, 0);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  Pipe pp;
  Cta c = begin<S>(t3_smem_raw, pp);
  const int Q0 = toff / 16 + tile * 8;
  const int nvQ = max(0, min(8, nQ - Q0));
  const int nb = nblocks(m, lmax);
  const int nbuf = nb * (NC == 1 ? 1 : 2);
  const int nst = 2 * nbuf;
  const int64_t base = alm_index(m, m, lmax);
  const int64_t gb0 = blockoff[m];
  const uint8_t* tab = reinterpret_cast<const uint8_t*>(table);
  bool ok = true;
  int mma_issued = 0, raw_issued = 0;

  if (warp < MMA_WARPS) {
    // ---- MMA issue: stage s reads A from staging buffer s >> 1 (position group s & 1 of it) and B
    // from operand buffer s % NB, into D[(s >> 1) & 1] (a D period = a staging buffer = 32 K values)
    const int acc = warp;
    const int p0 = acc, p1 = 1 - acc;  // spin s: parities of the F+ and F- K groups
    const uint32_t alb = NC == 1 ? u::POS8 : uint32_t(int(u::COMP) + (p1 - p0) * int(u::PAR));
    const uint32_t asb = NC == 1 ? u::R8 : 2u * u::POS8;
    for (int s = 0; s < nst && ok; ++s) {
      const int p = s >> 1, ls = s & 1, r = s >> 1;
      ok = wait(pp, pp.full + 8u * uint32_t(r % NR), uint32_t(r / NR) & 1u, err_flag);
      if (ok) ok = wait(pp, pp.op_full + 8u * uint32_t(s % NB), uint32_t(s / NB) & 1u, err_flag);
      if (ok && ls == 0 && p >= 2) ok = wait(pp, pp.d_free + 8u * uint32_t(p & 1), uint32_t((p >> 1) - 1) & 1u, err_flag);
      if (!ok) break;
      tc::fence_after_sync();
      const uint32_t a0 = c.sbase + S::raw(r % NR) +
                          (NC == 1 ? 2u * uint32_t(ls) * u::POS8 + uint32_t(acc) * u::PAR
                                   : uint32_t(ls) * u::POS8 + uint32_t(p0) * u::PAR);
      mma6(c.tmem + tcol_d(p & 1, acc), a0, alb, asb, c.sbase + S::b(s % NB, acc, 0), S::BT, idesc, ls == 0);
      tc::mma_commit_elect(pp.mma_done + 8u * uint32_t(s % NB));
      if (ls == 1) {
        tc::mma_commit_elect(pp.d_ready + 8u * uint32_t(p & 1));
        tc::mma_commit_elect(pp.raw_free + 8u * uint32_t(r % NR));
      }
      mma_issued = s + 1;
    }
  } else if (warp == COPY_WARP) {
    // ---- bulk copies of staging buffer r
    for (int r = 0; r < nbuf; ++r) {
      if (r >= NR) {
        ok = wait(pp, pp.raw_free + 8u * uint32_t(r % NR), uint32_t((r / NR) - 1) & 1u, err_flag);
        if (!ok) break;
      }
      const uint32_t bar = pp.full + 8u * uint32_t(r % NR);
      const uint32_t dst = c.sbase + S::raw(r % NR);
      if (NC == 1) {
        if (lane == 0) {
          tc::mbar_arrive_expect_tx(bar, uint32_t(nvQ) * u::UNIT);
          if (nvQ > 0)
            tc::bulk_g2s(dst, tab + (int64_t(gb0 + r) * nQ + Q0) * int64_t(u::UNIT), uint32_t(nvQ) * u::UNIT, bar);
        }
      } else {
        const int b = r >> 1, pp2 = r & 1;
        if (lane == 0) tc::mbar_arrive_expect_tx(bar, uint32_t(nvQ) * 2u * 2u * u::POS8);
        __syncwarp();  // the transaction count is expected before any copy lands
        const int qd = lane >> 1, r8 = lane & 1;
        if (lane < 16 && qd < nvQ)
          tc::bulk_g2s(dst + uint32_t(lane) * 2u * u::POS8,
                       tab + (int64_t(gb0 + b) * nQ + Q0 + qd) * int64_t(u::UNIT) + r8 * int64_t(u::R8) +
                           pp2 * 2 * int64_t(u::POS8),
                       2u * u::POS8, bar);
      }
      __syncwarp();
      raw_issued = r + 1;
    }
  } else if (warp >= PROD0 && warp < PROD0 + NPROD) {
    // ---- B operand producers: task pt < 4 gs = (map j, accumulator acc, K group kg): the 8 a_lm of its
    // K group as three BF16 planes (spin 0: rows re j, im gs + j; spin s: rows part gs + j, parts as
    // the FP32 kernels' X or Y combination)
    const int pt = tid - 32 * PROD0;
    const bool tv = pt < 4 * gs;
    const int j = tv ? pt % gs : 0, rest = tv ? pt / gs : 0;
    const int acc = rest & 1, kg = rest >> 1;
    const int par = NC == 1 ? acc : (kg == 0 ? acc : 1 - acc);
    double2 ab[8][NC];
    auto load = [&](int s) {
      int jpos0;  // first table position of the task's K group
      int b;
      if (NC == 1) { b = s >> 1; jpos0 = 16 * (s & 1) + 8 * kg; }
      else { b = s >> 2; jpos0 = 8 * (2 * ((s >> 1) & 1) + (s & 1)); }
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int l = m + LB * b + 2 * (jpos0 + i) + par;
        const bool v = tv && l <= lmax;
        const int64_t o = ((base + (l - m)) * B + b0 + j) * NC;
#pragma unroll
        for (int cc = 0; cc < NC; ++cc) ab[i][cc] = v ? almT[o + cc] : make_double2(0.0, 0.0);
      }
    };
    load(0);
    for (int s = 0; s < nst; ++s) {
      const int buf = s % NB;
      if (s >= NB) ok = wait(pp, pp.mma_done + 8u * uint32_t(buf), uint32_t((s / NB) - 1) & 1u, err_flag);
      if (!ok) break;
      if (tv) {
        const uint32_t pl0 = S::b(buf, acc, 0);
        if (NC == 1) {
          float re[8], im[8];
#pragma unroll
          for (int i = 0; i < 8; ++i) { re[i] = float(ab[i][0].x); im[i] = float(ab[i][0].y); }
          st_b8(c.smem, pl0, S::BT, j, kg, re);
          st_b8(c.smem, pl0, S::BT, gs + j, kg, im);
        } else {
          // F+ rows take X = -(G, C) (even spin) or Y = (C.im, -C.re, -G.im, G.re); F- rows the other one
          const bool use_x = (kg == 0) != (spin_odd != 0);
          float pv[4][8];
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            const float gr = float(ab[i][0].x), gi = float(ab[i][0].y);
            const float cr = float(ab[i][NC - 1].x), ci = float(ab[i][NC - 1].y);
            if (use_x) { pv[0][i] = -gr; pv[1][i] = -gi; pv[2][i] = -cr; pv[3][i] = -ci; }
            else { pv[0][i] = ci; pv[1][i] = -cr; pv[2][i] = -gi; pv[3][i] = gr; }
          }
#pragma unroll
          for (int part = 0; part < 4; ++part) st_b8(c.smem, pl0, S::BT, part * gs + j, kg, pv[part]);
        }
      }
      tc::fence_proxy_async();  // the operand stores, visible to the tensor core
      arrive(pp.op_full + 8u * uint32_t(buf));
      if (s + 1 < nst) load(s + 1);
    }
  } else if (warp >= DRAIN0) {
    const int npairs = nst >> 1;
    for (int p = 0; p < npairs; ++p) {
      ok = wait(pp, pp.d_ready + 8u * uint32_t(p & 1), uint32_t(p >> 1) & 1u, err_flag);
      if (!ok) break;
      tc::fence_after_sync();
      drain(c.tmem, warp, n, p);
      tc::fence_before_sync();
      arrive(pp.d_free + 8u * uint32_t(p & 1));
    }
  }
  tc::fence_before_sync();
  const bool failed = __syncthreads_or(!ok) != 0;
  tc::fence_after_sync();
  if (!failed) {
    // epilogue: TMEM lane t = ring 16 Q0 + t of the table; rows [north/south][lane][map][part] through
    // shared memory (free now), then every ring's row of gs maps with coalesced stores
    constexpr int RS = NMAX + 1;
    static_assert(2 * 128 * RS * 4 <= int(S::MISC_OFF), "epilogue rows exceed the free shared memory");
    float* rows = reinterpret_cast<float*>(c.smem);
    const int lq = warp & 3, cs = warp >> 2;
    const int tl = 32 * lq + lane;
#pragma unroll 1
    for (int cb = 16 * cs; cb < n; cb += 64) {
      float s0[16], s1[16];
      read_sum(c.tmem, 0, cb, s0);
      read_sum(c.tmem, 1, cb, s1);
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const int col = cb + q;
        if (col >= ncols) break;
        const int part = col / gs, jm = col % gs;
        const int pos = jm * 2 * NC + part;
        rows[tl * RS + pos] = s0[q] + s1[q];
        rows[(128 + tl) * RS + pos] = s0[q] - s1[q];
      }
    }
    __syncthreads();
    const int R = 2 * nrp - 1;
#pragma unroll 1
    for (int row = warp; row < 256; row += THREADS / 32) {
      const int ns = row >> 7, t = row & 127;
      const int rt = 16 * Q0 + t;  // table ring of TMEM lane t
      const int i = rt - toff;     // ring pair of the plan
      if (rt < toff || i >= nrp) continue;
      const int ring = ns == 0 ? i : R - 1 - i;
      if (ns == 1 && ring == i) continue;  // the equator has no south ring
      float* dst = reinterpret_cast<float*>(phase + ((int64_t(ring) * (mmax + 1) + m) * B + b0) * NC);
      const float* src = rows + row * RS;
      for (int pos = lane; pos < ncols; pos += 32) dst[pos] = src[pos];
    }
  } else if (lane == 0 && warp < MMA_WARPS && mma_issued > 0) {
    const int sp = mma_issued - 1;
    tc::mbar_wait_bounded(pp.mma_done + 8u * uint32_t(sp % NB), uint32_t(sp / NB) & 1u, WAIT_LIMIT);
  } else if (lane == 0 && warp == COPY_WARP) {
    for (int k = max(0, raw_issued - NR); k < raw_issued; ++k)
      tc::mbar_wait_bounded(pp.full + 8u * uint32_t(k % NR), uint32_t(k / NR) & 1u, WAIT_LIMIT);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(c.tmem, S::TMEM_COLS);
}


// ------------------------------------------------------------------ adjoint
// staging buffer = one stage: spin 0 the 8 pieces (block, ring half) of 3 KB of one slab, placed
// [half][block]; spin s the 4 pieces (block) of 6 KB of one ring half of a slab
constexpr uint32_t ADJ_RAW = 24576u;
constexpr int ADJ_NR = 6;

// phase [R][mmax+1][B][NC] complex64 of ring pairs [0, nrp) -> alm of map b at alm + b * out_stride
// ([NC][nalm] complex128, times scale and lscale[comp][idx] when given), for the maps [b0, b0 + gs)
// of each group.  grid.x = map group + G * (entry of the (m, first block) work list)
template <int NC>
__global__ void __launch_bounds__(THREADS, 1) adj_kernel(const uint16_t* __restrict__ table,
                                                         const int64_t* __restrict__ blockoff, int nQ, int toff,
                                                         int nrp, int lmax, int mmax, const float2* __restrict__ phase,
                                                         double2* __restrict__ alm, int B, int gsize, int ngroups,
                                                         const int2* __restrict__ work, int64_t nalm, double scale,
                                                         int spin_odd, int64_t out_stride,
                                                         const double* __restrict__ lscale,
                                                         int* __restrict__ err_flag) {
  using u = U<NC>;
  using S = Smem<ADJ_RAW, ADJ_NR>;
  constexpr int NR = S::NR;
  extern __shared__ uint8_t t3_smem_raw[];
  int bid = blockIdx.x;
  const int grp = bid % ngroups; bid /= ngroups;
  const int2 wk = work[bid];  // (m, first block of the group of 4)
  const int m = wk.x, bb = wk.y;
  const int b0 = grp * gsize;
  const int gs = min(gsize, B - b0);
  const int ncols = 2 * NC * gs;
  const int n = round16(ncols);
  const uint32_t idesc = tc::idesc_bf16(128, n, 0, 0);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  Pipe pp;
  Cta c = begin<S>(t3_smem_raw, pp);
  const int nb = nblocks(m, lmax);
  const int nblk = min(4, nb - bb);
  const int R = 2 * nrp - 1;
  const int rt_begin = toff & ~15, rt_end = toff + nrp;
  const int nslab = (rt_end - rt_begin + 15) / 16;
  const int nst = NC == 1 ? nslab : 2 * nslab;
  const int npairs = (nst + 1) >> 1;  // D periods (the last may hold one stage)
  const int64_t gb0 = blockoff[m] + bb;
  const uint8_t* tab = reinterpret_cast<const uint8_t*>(table);
  bool ok = true;
  int mma_issued = 0, raw_issued = 0;

  if (warp < MMA_WARPS) {
    // ---- MMA issue: stage st (A K-major from staging buffer st % NR, B from operand buffer st % NB)
    const int acc = warp;
    const uint32_t alb = NC == 1 ? 4u * u::R8 : u::COMP;  // K groups: ring halves / F+ then F-
    const uint32_t asb = u::POS8;                          // M groups: 8 positions (4 per block)
    for (int st = 0; st < nst; ++st) {
      const int p = st >> 1;
      ok = wait(pp, pp.full + 8u * uint32_t(st % NR), uint32_t(st / NR) & 1u, err_flag);
      if (ok) ok = wait(pp, pp.op_full + 8u * uint32_t(st % NB), uint32_t(st / NB) & 1u, err_flag);
      if (ok && (st & 1) == 0 && p >= 2) ok = wait(pp, pp.d_free + 8u * uint32_t(p & 1), uint32_t((p >> 1) - 1) & 1u, err_flag);
      if (!ok) break;
      tc::fence_after_sync();
      const uint32_t a0 = c.sbase + S::raw(st % NR) + uint32_t(acc) * u::PAR;
      mma6(c.tmem + tcol_d(p & 1, acc), a0, alb, asb, c.sbase + S::b(st % NB, acc, 0), S::BT, idesc, (st & 1) == 0);
      tc::mma_commit_elect(pp.mma_done + 8u * uint32_t(st % NB));
      tc::mma_commit_elect(pp.raw_free + 8u * uint32_t(st % NR));
      if ((st & 1) || st == nst - 1) tc::mma_commit_elect(pp.d_ready + 8u * uint32_t(p & 1));
      mma_issued = st + 1;
    }
  } else if (warp == COPY_WARP) {
    for (int st = 0; st < nst; ++st) {
      if (st >= NR) {
        ok = wait(pp, pp.raw_free + 8u * uint32_t(st % NR), uint32_t((st / NR) - 1) & 1u, err_flag);
        if (!ok) break;
      }
      const int Q = rt_begin / 16 + (NC == 1 ? st : st >> 1);
      const uint32_t bar = pp.full + 8u * uint32_t(st % NR);
      const uint32_t dst = c.sbase + S::raw(st % NR);
      if (NC == 1) {
        if (lane == 0) tc::mbar_arrive_expect_tx(bar, uint32_t(nblk) * 2u * u::R8);
        __syncwarp();
        const int bk = lane >> 1, r8 = lane & 1;
        if (lane < 8 && bk < nblk)
          tc::bulk_g2s(dst + uint32_t(r8) * 4u * u::R8 + uint32_t(bk) * u::R8,
                       tab + (int64_t(gb0 + bk) * nQ + Q) * int64_t(u::UNIT) + r8 * int64_t(u::R8), u::R8, bar);
      } else {
        const int r8 = st & 1;
        if (lane == 0) tc::mbar_arrive_expect_tx(bar, uint32_t(nblk) * u::R8);
        __syncwarp();
        if (lane < nblk)
          tc::bulk_g2s(dst + uint32_t(lane) * u::R8,
                       tab + (int64_t(gb0 + lane) * nQ + Q) * int64_t(u::UNIT) + r8 * int64_t(u::R8), u::R8, bar);
      }
      __syncwarp();
      raw_issued = st + 1;
    }
  } else if (warp >= PROD0 && warp < PROD0 + NPROD) {
    // ---- B operand producers.  spin 0: task pt < 2 gs = (map j, ring half kg): the ring sums
    // (accumulator 0: N + S) and differences (accumulator 1: N - S) of its 8 rings, re and im rows.
    // spin s: task pt < 4 gs = (map j, accumulator acc, component kg: F+ / F-): combo k = kg ? 1 - acc
    // : acc of the (Q, U) of its 8 rings, four part rows (X or Y as the FP32 kernels)
    const int pt = tid - 32 * PROD0;
    const bool tv = pt < (NC == 1 ? 2 : 4) * gs;
    const int j = tv ? pt % gs : 0, rest = tv ? pt / gs : 0;
    const int acc = NC == 1 ? 0 : (rest & 1);
    const int kg = NC == 1 ? rest : (rest >> 1);
    float4 pn[8], pv[8];  // spin 0 uses .x .y only
    auto load = [&](int st) {
      const int rs0 = rt_begin + (NC == 1 ? 16 * st + 8 * kg : 16 * (st >> 1) + 8 * (st & 1));
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int ip = rs0 + i - toff;
        const bool in = tv && ip >= 0 && ip < nrp;
        const int rsth = R - 1 - ip;
        const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
        if (NC == 1) {
          const float2 a = in ? phase[(int64_t(ip) * (mmax + 1) + m) * B + b0 + j] : make_float2(0.f, 0.f);
          const float2 bv = (in && rsth != ip) ? phase[(int64_t(rsth) * (mmax + 1) + m) * B + b0 + j] : make_float2(0.f, 0.f);
          pn[i] = make_float4(a.x, a.y, 0.f, 0.f);
          pv[i] = make_float4(bv.x, bv.y, 0.f, 0.f);
        } else {
          const float4* ph4 = reinterpret_cast<const float4*>(phase);
          pn[i] = in ? ph4[(int64_t(ip) * (mmax + 1) + m) * B + b0 + j] : z;
          pv[i] = (in && rsth != ip) ? ph4[(int64_t(rsth) * (mmax + 1) + m) * B + b0 + j] : z;
        }
      }
    };
    load(0);
    for (int st = 0; st < nst; ++st) {
      const int buf = st % NB;
      if (st >= NB) ok = wait(pp, pp.mma_done + 8u * uint32_t(buf), uint32_t((st / NB) - 1) & 1u, err_flag);
      if (!ok) break;
      if (tv) {
        if (NC == 1) {
#pragma unroll
          for (int a = 0; a < 2; ++a) {
            float re[8], im[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) {
              re[i] = a == 0 ? pn[i].x + pv[i].x : pn[i].x - pv[i].x;
              im[i] = a == 0 ? pn[i].y + pv[i].y : pn[i].y - pv[i].y;
            }
            st_b8(c.smem, S::b(buf, a, 0), S::BT, j, kg, re);
            st_b8(c.smem, S::b(buf, a, 0), S::BT, gs + j, kg, im);
          }
        } else {
          // columns (G.re, G.im, C.re, C.im); combo k (0: N + S, 1: N - S) of the rings' (Q, U):
          // X(k) = (-Q.re, -Q.im, -U.re, -U.im), Y(k) = (U.im, -U.re, -Q.im, Q.re);
          // even spin: F+ rows X(acc), F- rows Y(1 - acc); odd spin: F+ rows Y(acc), F- rows X(1 - acc)
          const int k = kg == 0 ? acc : 1 - acc;
          const bool use_x = (kg == 0) != (spin_odd != 0);
          float pr[4][8];
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            const float4 cv = k == 0 ? make_float4(pn[i].x + pv[i].x, pn[i].y + pv[i].y, pn[i].z + pv[i].z, pn[i].w + pv[i].w)
                                     : make_float4(pn[i].x - pv[i].x, pn[i].y - pv[i].y, pn[i].z - pv[i].z, pn[i].w - pv[i].w);
            if (use_x) { pr[0][i] = -cv.x; pr[1][i] = -cv.y; pr[2][i] = -cv.z; pr[3][i] = -cv.w; }
            else { pr[0][i] = cv.w; pr[1][i] = -cv.z; pr[2][i] = -cv.y; pr[3][i] = cv.x; }
          }
#pragma unroll
          for (int part = 0; part < 4; ++part) st_b8(c.smem, S::b(buf, acc, 0), S::BT, part * gs + j, kg, pr[part]);
        }
      }
      tc::fence_proxy_async();
      arrive(pp.op_full + 8u * uint32_t(buf));
      if (st + 1 < nst) load(st + 1);
    }
  } else if (warp >= DRAIN0) {
    for (int p = 0; p < npairs; ++p) {
      ok = wait(pp, pp.d_ready + 8u * uint32_t(p & 1), uint32_t(p >> 1) & 1u, err_flag);
      if (!ok) break;
      tc::fence_after_sync();
      drain(c.tmem, warp, n, p);
      tc::fence_before_sync();
      arrive(pp.d_free + 8u * uint32_t(p & 1));
    }
  }
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
      const int l = m + LB * (bb + blk) + 2 * lane + acc;
      const bool in = blk < nblk && l <= lmax;
      const int64_t idx = alm_index(l, m, lmax);
#pragma unroll 1
      for (int cb = 16 * cs; cb < n; cb += 64) {
        float sm[16];
        read_sum(c.tmem, acc, cb, sm);
        if (!in) continue;
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
  } else if (failed && lane == 0 && warp < MMA_WARPS && mma_issued > 0) {
    const int sp = mma_issued - 1;
    tc::mbar_wait_bounded(pp.mma_done + 8u * uint32_t(sp % NB), uint32_t(sp / NB) & 1u, WAIT_LIMIT);
  } else if (failed && lane == 0 && warp == COPY_WARP) {
    for (int k = max(0, raw_issued - NR); k < raw_issued; ++k)
      tc::mbar_wait_bounded(pp.full + 8u * uint32_t(k % NR), uint32_t(k / NR) & 1u, WAIT_LIMIT);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(c.tmem, S::TMEM_COLS);
}

}  // namespace t3
}  // namespace ps

// ------------------------------------------------------------------ host side
namespace ps {
namespace {
int t3_smem_attr(const void* fn, int bytes) {
  return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) == cudaSuccess ? PS_OK
                                                                                                       : PS_ERR_CUDA;
}
int t3_group_size(int B, int spin, int& ngroups) {
  const int cap = spin == 0 ? t3::NMAX / 2 : t3::NMAX / 4;
  ngroups = (B + cap - 1) / cap;
  return (B + ngroups - 1) / ngroups;
}
}  // namespace

size_t tab3_bytes(int Rh, int lmax, int mmax, int spin) {
  return size_t(tab_total_blocks(lmax, mmax)) * size_t(t3::nslabs(Rh)) *
         size_t(spin == 0 ? t3::U<1>::UNIT : t3::U<2>::UNIT);
}

int launch_tab3_gen(const Plan& P, int spin, const int64_t* d_blockoff, uint16_t* table, cudaStream_t st) {
  const int nQ = t3::nslabs(P.Rh);
  dim3 grid(nQ * 16 / t3::TILE, P.mmax + 1);
  if (spin == 0) {
    const int smem = 8 * int(t3::U<1>::UNIT);
    if (t3_smem_attr((const void*)t3::gen_kernel<1>, smem)) return PS_ERR_CUDA;
    t3::gen_kernel<1><<<grid, t3::GEN_THREADS, smem, st>>>(P.d_rings, P.d_mnorm0, nullptr, P.Rh, P.lmax, 0, d_blockoff,
                                                          nQ, table);
  } else {
    if (!P.d_seed[spin]) return PS_ERR_INVALID;
    const int smem = 8 * int(t3::U<2>::UNIT);
    if (t3_smem_attr((const void*)t3::gen_kernel<2>, smem)) return PS_ERR_CUDA;
    t3::gen_kernel<2><<<grid, t3::GEN_THREADS, smem, st>>>(P.d_rings, nullptr, P.d_seed[spin], P.Rh, P.lmax, spin,
                                                          d_blockoff, nQ, table);
  }
  PS_LAUNCH_CHECK();
  return PS_OK;
}

// the table of ring pairs [toff, toff + P.Rh) of a plan whose table has Rh_table ring pairs
int launch_tab3_synth(const Plan& P, const uint16_t* table, const int64_t* d_blockoff, int Rh_table, int toff,
                      const double2* almT, float2* phase, int B, int spin, int* err_flag, cudaStream_t st) {
  const double flops = double(spin == 0 ? 4 : 16) * double(P.Rh) * double(P.nalm) * B;
  const double bytes = double(tab3_bytes(Rh_table, P.lmax, P.mmax, spin)) * double(P.Rh) / double(Rh_table) +
                       double(B) * (spin == 0 ? 1 : 2) * (16.0 * P.nalm + 8.0 * P.R * (P.mmax + 1));
  StatScope sc(PS_K_LEG_SYNTH, flops, bytes, st);
  int ngroups = 1;
  const int gsize = t3_group_size(B, spin, ngroups);
  const int ntiles = ((toff & 15) + P.Rh + t3::TILE - 1) / t3::TILE;
  const int nQ = t3::nslabs(Rh_table);
  const int64_t nblk = int64_t(ngroups) * ntiles * (P.mmax + 1);
  if (nblk > 0x7fffffff) return PS_ERR_UNSUPPORTED;
  using S = t3::Smem<t3::SYN_RAW, t3::SYN_NR>;
  const int smem = int(S::DYN);
  if (spin == 0) {
    if (t3_smem_attr((const void*)t3::synth_kernel<1>, smem)) return PS_ERR_CUDA;
    t3::synth_kernel<1><<<unsigned(nblk), t3::THREADS, smem, st>>>(table, d_blockoff, nQ, toff, P.Rh, P.lmax, P.mmax,
                                                                   almT, phase, B, gsize, ngroups, ntiles, 0, err_flag);
  } else {
    if (t3_smem_attr((const void*)t3::synth_kernel<2>, smem)) return PS_ERR_CUDA;
    t3::synth_kernel<2><<<unsigned(nblk), t3::THREADS, smem, st>>>(table, d_blockoff, nQ, toff, P.Rh, P.lmax, P.mmax,
                                                                   almT, phase, B, gsize, ngroups, ntiles, spin & 1,
                                                                   err_flag);
  }
  PS_LAUNCH_CHECK();
  return PS_OK;
}

int launch_tab3_adj(const Plan& P, const uint16_t* table, const int64_t* d_blockoff, const int2* d_work, int nwork,
                    int Rh_table, int toff, const float2* phase, double2* alm, int B, int spin, double scale,
                    int64_t out_stride, const double* lscale, int* err_flag, cudaStream_t st) {
  const double flops = double(spin == 0 ? 4 : 16) * double(P.Rh) * double(P.nalm) * B;
  const double bytes = double(tab3_bytes(Rh_table, P.lmax, P.mmax, spin)) * double(P.Rh) / double(Rh_table) +
                       double(B) * (spin == 0 ? 1 : 2) * (16.0 * P.nalm + 8.0 * P.R * (P.mmax + 1));
  StatScope sc(PS_K_LEG_ADJOINT, flops, bytes, st);
  int ngroups = 1;
  const int gsize = t3_group_size(B, spin, ngroups);
  const int nQ = t3::nslabs(Rh_table);
  const int64_t nblk = int64_t(ngroups) * nwork;
  if (nblk > 0x7fffffff) return PS_ERR_UNSUPPORTED;
  // spin s phases are read as float4 (Q, U of one map)
  if (spin != 0 && (reinterpret_cast<uintptr_t>(phase) & 15u)) return PS_ERR_INVALID;
  using S = t3::Smem<t3::ADJ_RAW, t3::ADJ_NR>;
  const int smem = int(S::DYN);
  if (spin == 0) {
    if (t3_smem_attr((const void*)t3::adj_kernel<1>, smem)) return PS_ERR_CUDA;
    t3::adj_kernel<1><<<unsigned(nblk), t3::THREADS, smem, st>>>(table, d_blockoff, nQ, toff, P.Rh, P.lmax, P.mmax,
                                                                 phase, alm, B, gsize, ngroups, d_work, P.nalm, scale,
                                                                 0, out_stride, lscale, err_flag);
  } else {
    if (t3_smem_attr((const void*)t3::adj_kernel<2>, smem)) return PS_ERR_CUDA;
    t3::adj_kernel<2><<<unsigned(nblk), t3::THREADS, smem, st>>>(table, d_blockoff, nQ, toff, P.Rh, P.lmax, P.mmax,
                                                                 phase, alm, B, gsize, ngroups, d_work, P.nalm, scale,
                                                                 spin & 1, out_stride, lscale, err_flag);
  }
  PS_LAUNCH_CHECK();
  return PS_OK;
}

}  // namespace ps
