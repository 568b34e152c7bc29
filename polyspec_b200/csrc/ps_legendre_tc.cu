// Mixed-precision Legendre stage of the synthesis on the 5th-generation tensor
// cores (tcgen05, kind::tf32, accumulators in TMEM).
//
// For order m and a tile of 128 ring pairs, with l split by the parity of l+m:
//   D_p[ring, n] = sum_{l : (l+m)%2 = p} Lam[ring, l] * A[l, n]     (p = 0, 1)
// where n runs over the real and imaginary parts of the maps' a_lm (spin 0)
// or of (G, C) (spin s, with Lam = F+ and F- as two A operands).  The north
// ring takes D_0 + D_1, the mirror ring D_0 - D_1 (and the F-/F+ sign rules of
// the HEALPix spin conventions for spin s).
//
// Lam tiles are generated on the fly: one thread per ring runs the FP64
// recurrence (scaled seeds as in the FP64 kernels), rounds each value to FP32
// and splits it into two TF32 parts hi + lo (K-major operand, 8-row x 16-byte
// core matrices, no swizzle).  The a_lm of the chunk are split the same way.
// Three tcgen05.mma per parity (hi*hi + hi*lo + lo*hi) accumulate one chunk in
// FP32 in TMEM; after each chunk every thread moves its TMEM row into FP32
// registers (round-to-nearest adds) and the next chunk starts a fresh TMEM
// accumulation.  The tensor cores' FP32 accumulation truncates, so a single
// accumulator running over all l (about 770 MMA steps at lmax 2048) biases the
// result towards zero by ~1e-5 relative; one chunk (3 steps) keeps that bias
// below 1e-6.  Chunks of 16 l (8 per parity) keep a CTA's shared memory small
// so that several CTAs share an SM and hide the latency of the recurrence
// chains; two stages of tiles let the tensor cores work on chunk c-1 while the
// threads generate chunk c (a tcgen05.commit per stage on its mbarrier tells
// when the chunk's MMAs are done), and the chunk is drained just before the
// next one is issued.  The next chunk's a_lm and recurrence coefficients are
// fetched while the current chunk is generated.  Every mbarrier wait is
// bounded; on expiry the kernel raises the plan's error flag, waits once more
// (bounded) for its MMAs and frees its TMEM.
#include "ps_common.cuh"
#include "ps_stats.cuh"
#include "ps_tc.cuh"

namespace ps {

constexpr int TC_RT = 128;  // ring pairs per CTA (MMA M)
constexpr int TC_LC = 16;   // l per chunk (8 of each parity = one MMA K step)
constexpr uint32_t TC_WAIT_LIMIT = 1u << 24;

__device__ __forceinline__ void seed0_tc(int m, double sth, double mnorm, double& v, int& k) {
  Scaled s = smul(spow(sth, m), snorm(mnorm));
  to_kscale(s, v, k);
  if (m & 1) v = -v;
}

__device__ __forceinline__ void seedS_tc(int m, int s, const RingInfo& g, SeedNorm nrm, double& f, double& gg,
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

__device__ __forceinline__ void split_tf32(double x, float& hi, float& lo) {
  const float f = float(x);
  hi = tc::tf32_rna(f);
  lo = tc::tf32_rna(f - hi);
}

// K-major operand without swizzle: core matrix (row/8, kc) of 8 rows x 16 bytes
// at ((row/8)*2 + kc)*128; leading (K) byte offset 128, stride (8-row) 256.
__device__ __forceinline__ uint32_t core_off(int row, int kc) {
  return uint32_t(((row >> 3) * 2 + kc) * 128 + (row & 7) * 16);
}
__device__ __forceinline__ uint64_t desc_k8(uint32_t saddr) {
  uint64_t d = 0;
  d |= uint64_t((saddr >> 4) & 0x3FFFu);
  d |= uint64_t(128u >> 4) << 16;  // leading byte offset
  d |= uint64_t(256u >> 4) << 32;  // stride byte offset
  d |= uint64_t(1) << 46;          // descriptor version
  return d;                        // layout type 0: no swizzle
}

// Shared-memory plan (offsets from a 1024-byte aligned base):
//   stage st: A[op][p][h] 4 KB each, B[p][h] N*32 bytes each
//   coefficient buffers [2][3][TC_LC] doubles, 2 mbarriers, TMEM slot
template <int NOPS, int N>
struct TcSmem {
  static constexpr uint32_t A_BYTES = TC_RT * 8 * 4;
  static constexpr uint32_t B_BYTES = N * 8 * 4;
  static constexpr uint32_t STAGE = NOPS * 4 * A_BYTES + 4 * B_BYTES;
  static constexpr uint32_t COEF_OFF = 2 * STAGE;
  static constexpr uint32_t MISC_OFF = COEF_OFF + 2 * 3 * TC_LC * 8;
  static constexpr uint32_t TOTAL = MISC_OFF + 64;
  static constexpr uint32_t DYN = TOTAL + 1024;
  __device__ static uint32_t a(int st, int op, int p, int h) { return st * STAGE + ((op * 2 + p) * 2 + h) * A_BYTES; }
  __device__ static uint32_t b(int st, int p, int h) { return st * STAGE + NOPS * 4 * A_BYTES + (p * 2 + h) * B_BYTES; }
};

template <int NOPS, int N>
__device__ __forceinline__ void issue_stage(uint32_t sbase, int st, uint32_t tmem) {
  constexpr uint32_t idesc = tc::idesc_tf32(128, N, 0, 0);
  using S = TcSmem<NOPS, N>;
#pragma unroll
  for (int op = 0; op < NOPS; ++op)
#pragma unroll
    for (int p = 0; p < 2; ++p) {
      const uint32_t d = tmem + uint32_t((op * 2 + p) * N);
      const uint64_t a_hi = desc_k8(sbase + S::a(st, op, p, 0)), a_lo = desc_k8(sbase + S::a(st, op, p, 1));
      const uint64_t b_hi = desc_k8(sbase + S::b(st, p, 0)), b_lo = desc_k8(sbase + S::b(st, p, 1));
      tc::mma_tf32(d, a_hi, b_hi, idesc, 0u);  // fresh accumulation per chunk
      tc::mma_tf32(d, a_hi, b_lo, idesc, 1u);
      tc::mma_tf32(d, a_lo, b_hi, idesc, 1u);
    }
}

// four values of ring r's row (one 16-byte core row)
__device__ __forceinline__ void put_a4(uint8_t* smem, uint32_t off, int r, int kc, float a, float b, float c,
                                       float d) {
  *reinterpret_cast<float4*>(smem + off + core_off(r, kc)) = make_float4(a, b, c, d);
}

// =====================================================================
// One kernel for spin 0 (NOPS = 1) and spin s (NOPS = 2).
//   spin 0: almT [nalm][B] complex128; phase [R][mmax+1][B] complex64; N = 2 BC
//   spin s: almT [nalm][B][2]; phase [R][mmax+1][B][2]; N = 4 BC
// grid (ceil(Rh/128), mmax+1, ceil(B/BC)), 128 threads
template <int NOPS, int BC>
__global__ void __launch_bounds__(TC_RT) synth_tc(const RingInfo* __restrict__ rings,
                                                   const double* __restrict__ mnorm,
                                                   const SeedNorm* __restrict__ seednorm,
                                                   const double2* __restrict__ almT, float2* __restrict__ phase,
                                                   int R, int Rh, int lmax, int mmax, int B, int spin,
                                                   int* __restrict__ err_flag) {
  constexpr int NCOMP = NOPS;        // complex inputs per (l, map): a or (G, C)
  constexpr int N = 2 * NCOMP * BC;  // B-tile rows: (re, im) of each complex input of each map
  constexpr uint32_t NCOLS_NEED = 2 * NOPS * N;
  constexpr uint32_t NCOLS = NCOLS_NEED <= 32 ? 32 : NCOLS_NEED <= 64 ? 64 : NCOLS_NEED <= 128 ? 128
                            : NCOLS_NEED <= 256 ? 256 : 512;
  using S = TcSmem<NOPS, N>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const uint32_t sbase = tc::smem_u32(smem);
  double* s_coef = reinterpret_cast<double*>(smem + S::COEF_OFF);  // [2][3][TC_LC]
  uint64_t* s_mbar = reinterpret_cast<uint64_t*>(smem + S::MISC_OFF);
  uint32_t* s_tmem = reinterpret_cast<uint32_t*>(smem + S::MISC_OFF + 16);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m = blockIdx.y;
  const int rp = blockIdx.x * TC_RT + tid;
  const int b0 = blockIdx.z * BC;
  const int lmin = NOPS == 1 ? m : max(m, spin);

  if (warp == 0) {
    tc::tmem_alloc(tc::smem_u32(s_tmem), NCOLS);
    tc::tmem_relinquish();
  }
  if (tid == 0) {
    tc::mbar_init(tc::smem_u32(&s_mbar[0]), 1);
    tc::mbar_init(tc::smem_u32(&s_mbar[1]), 1);
  }

  // recurrence coefficients of the chunk starting at l0 into buffer `buf`:
  //   spin 0: (a, b) stepping lam_l -> lam_{l+1}, l = l0 + t;  spin s: (A, D, C) stepping l -> l+1
  auto coefs = [&](int l0, int buf) {
    if (tid < TC_LC) {
      double c0 = 0.0, c1 = 0.0, c2 = 0.0;
      if (NOPS == 1) {
        const int l = l0 + tid + 1;
        if (l <= lmax) {
          const double mm = double(m) * m;
          c0 = sqrt((4.0 * l * l - 1.0) / (double(l) * l - mm));
          if (l >= m + 2) c1 = c0 / sqrt((4.0 * (l - 1.0) * (l - 1.0) - 1.0) / ((l - 1.0) * (l - 1.0) - mm));
        }
      } else {
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
      s_coef[(buf * 3 + 0) * TC_LC + tid] = c0;
      s_coef[(buf * 3 + 1) * TC_LC + tid] = c1;
      s_coef[(buf * 3 + 2) * TC_LC + tid] = c2;
    }
  };
  const int64_t base = alm_index(m, m, lmax);
  // B-tile items: one 16-byte core row = 4 l of one real component.  Item
  // idx = (p*2 + kc)*N + n covers row n (map column), parity p, K positions
  // 4kc..4kc+3, i.e. l = l0 + p + 2 (4 kc + i), i = 0..3; eight consecutive
  // items fill one core matrix, so the 16-byte stores are conflict-free.
  constexpr int NITEM = 4 * N;
  constexpr int IPT = (NITEM + TC_RT - 1) / TC_RT;
  double pre[IPT][4];
  auto fetch = [&](int l0) {
#pragma unroll
    for (int it = 0; it < IPT; ++it) {
      const int idx = tid + it * TC_RT;
      const int n = idx % N, pk = idx / N, p = pk >> 1, kc = pk & 1;
      const int part = n & 1;
      const int bi = n / (2 * NCOMP), cc = (n >> 1) % NCOMP;
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int l = l0 + p + 2 * (4 * kc + i);
        double v = 0.0;
        if (idx < NITEM && l <= lmax && b0 + bi < B) {
          const double2 a = almT[((base + (l - m)) * B + b0 + bi) * NCOMP + cc];
          v = part ? a.y : a.x;
        }
        pre[it][i] = v;
      }
    }
  };

  coefs(m, 0);
  fetch(m);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *s_tmem;

  // recurrence state of this thread's ring
  const bool active = rp < Rh;
  const RingInfo g = rings[active ? rp : 0];
  const double x = g.z;
  double f = 0.0, fp = 0.0, gg = 0.0, gp = 0.0, sf = 0.0, sg = 0.0;
  int k = 0;
  if (NOPS == 1) {
    seed0_tc(m, g.sth, mnorm[m], f, k);
  } else {
    seedS_tc(m, spin, g, seednorm[m], sf, sg, k);
  }
  if (!active) { f = 0.0; sf = 0.0; sg = 0.0; k = 0; }

  const int nchunks = (lmax - m) / TC_LC + 1;
  uint32_t ph[2] = {0u, 0u};
  bool ok = true;
  // FP32 running sums of this thread's TMEM row (all D regions)
  constexpr int NSUM = int(NCOLS_NEED);
  float acc[NSUM];
#pragma unroll
  for (int q = 0; q < NSUM; ++q) acc[q] = 0.f;
  const uint32_t lane_addr = tmem + (uint32_t(warp * 32) << 16);
  // wait for the MMAs of chunk cc (committed on mbarrier cc & 1) and add D to acc
  auto drain = [&](int cc) -> bool {
    const int sb = cc & 1;
    if (!__syncthreads_and(tc::mbar_wait_bounded(tc::smem_u32(&s_mbar[sb]), ph[sb], TC_WAIT_LIMIT))) return false;
    ph[sb] ^= 1u;
    tc::fence_after_sync();
#pragma unroll
    for (int cb = 0; cb < NSUM; cb += 16) {
      float v[16];
      tc::tmem_ld16(lane_addr + cb, v);
      tc::tmem_ld_wait();
#pragma unroll
      for (int q = 0; q < 16; ++q) acc[cb + q] += v[q];
    }
    tc::fence_before_sync();
    return true;
  };
  for (int c = 0; c < nchunks; ++c) {
    const int st = c & 1;
    const int l0 = m + c * TC_LC;
    // stage st was read by the MMAs of chunk c-2, drained (and so finished) in iteration c-1
    // B tiles of this chunk from the prefetched a_lm (l0 + m even: even l - l0 -> parity 0)
#pragma unroll
    for (int it = 0; it < IPT; ++it) {
      const int idx = tid + it * TC_RT;
      if (idx < NITEM) {
        const int n = idx % N, pk = idx / N, p = pk >> 1, kc = pk & 1;
        float h[4], lo[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) split_tf32(pre[it][i], h[i], lo[i]);
        *reinterpret_cast<float4*>(smem + S::b(st, p, 0) + core_off(n, kc)) = make_float4(h[0], h[1], h[2], h[3]);
        *reinterpret_cast<float4*>(smem + S::b(st, p, 1) + core_off(n, kc)) =
            make_float4(lo[0], lo[1], lo[2], lo[3]);
      }
    }
    if (c + 1 < nchunks) {
      fetch(l0 + TC_LC);
      coefs(l0 + TC_LC, st ^ 1);
    }
    // A tiles: 16 recurrence steps of this thread's ring
    const double* c0 = s_coef + (st * 3 + 0) * TC_LC;
    const double* c1 = s_coef + (st * 3 + 1) * TC_LC;
    const double* c2 = s_coef + (st * 3 + 2) * TC_LC;
    if (NOPS == 1) {
      float hv[TC_LC], lv[TC_LC];
#pragma unroll
      for (int j = 0; j < TC_LC; ++j) {
        const double val = (k == 0 && l0 + j <= lmax) ? f : 0.0;
        split_tf32(val, hv[j], lv[j]);
        const double nxt = c0[j] * x * f - c1[j] * fp;
        fp = f;
        f = nxt;
        if (k < 0 && fabs(f) > PS_FTHRESH) { f *= PS_FSMALL; fp *= PS_FSMALL; ++k; }
      }
#pragma unroll
      for (int p = 0; p < 2; ++p) {
        put_a4(smem, S::a(st, 0, p, 0), tid, 0, hv[p], hv[p + 2], hv[p + 4], hv[p + 6]);
        put_a4(smem, S::a(st, 0, p, 0), tid, 1, hv[p + 8], hv[p + 10], hv[p + 12], hv[p + 14]);
        put_a4(smem, S::a(st, 0, p, 1), tid, 0, lv[p], lv[p + 2], lv[p + 4], lv[p + 6]);
        put_a4(smem, S::a(st, 0, p, 1), tid, 1, lv[p + 8], lv[p + 10], lv[p + 12], lv[p + 14]);
      }
    } else {
      float ph_[TC_LC], pl_[TC_LC], mh_[TC_LC], ml_[TC_LC];
#pragma unroll
      for (int j = 0; j < TC_LC; ++j) {
        const int l = l0 + j;
        if (l == lmin) { f = sf; gg = sg; fp = 0.0; gp = 0.0; }
        const bool use = (k == 0) && (l <= lmax);
        split_tf32(use ? 0.5 * (f + gg) : 0.0, ph_[j], pl_[j]);
        split_tf32(use ? 0.5 * (f - gg) : 0.0, mh_[j], ml_[j]);
        const double ax = c0[j] * x;
        const double fn = (ax + c1[j]) * f - c2[j] * fp;
        const double gn = (ax - c1[j]) * gg - c2[j] * gp;
        fp = f; f = fn; gp = gg; gg = gn;
        if (k < 0 && fmax(fabs(f), fabs(gg)) > PS_FTHRESH) {
          f *= PS_FSMALL; fp *= PS_FSMALL; gg *= PS_FSMALL; gp *= PS_FSMALL; ++k;
        }
      }
#pragma unroll
      for (int p = 0; p < 2; ++p)
#pragma unroll
        for (int kc = 0; kc < 2; ++kc) {
          const int j0 = p + 8 * kc;
          put_a4(smem, S::a(st, 0, p, 0), tid, kc, ph_[j0], ph_[j0 + 2], ph_[j0 + 4], ph_[j0 + 6]);
          put_a4(smem, S::a(st, 0, p, 1), tid, kc, pl_[j0], pl_[j0 + 2], pl_[j0 + 4], pl_[j0 + 6]);
          put_a4(smem, S::a(st, 1, p, 0), tid, kc, mh_[j0], mh_[j0 + 2], mh_[j0 + 4], mh_[j0 + 6]);
          put_a4(smem, S::a(st, 1, p, 1), tid, kc, ml_[j0], ml_[j0 + 2], ml_[j0 + 4], ml_[j0 + 6]);
        }
    }
    // chunk c-1 must leave TMEM before chunk c's MMAs overwrite it
    if (c >= 1 && !drain(c - 1)) {
      ok = false;
      break;
    }
    tc::fence_proxy_async();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
      issue_stage<NOPS, N>(sbase, st, tmem);
      tc::mma_commit(tc::smem_u32(&s_mbar[st]));
    }
  }
  if (ok) ok = drain(nchunks - 1);
  if (!ok) {
    // the last commit arrives once every MMA of the CTA has completed
    const int stl = (nchunks - 1) & 1;
    if (tid == 0) atomicExch(err_flag, 1);
    tc::mbar_wait_bounded(tc::smem_u32(&s_mbar[stl]), ph[stl], TC_WAIT_LIMIT);
  } else {
    const int ring = blockIdx.x * TC_RT + warp * 32 + lane;
    const int rs = R - 1 - ring;
    if (NOPS == 1) {
#pragma unroll
      for (int cb = 0; cb < N; cb += 16) {
        const float* e = acc + cb;
        const float* o = acc + N + cb;
        if (ring < Rh) {
#pragma unroll
          for (int q = 0; q < 16; q += 2) {
            const int bi = (cb + q) >> 1;
            if (b0 + bi < B) {
              phase[(int64_t(ring) * (mmax + 1) + m) * B + b0 + bi] = make_float2(e[q] + o[q], e[q + 1] + o[q + 1]);
              if (rs != ring)
                phase[(int64_t(rs) * (mmax + 1) + m) * B + b0 + bi] =
                    make_float2(e[q] - o[q], e[q + 1] - o[q + 1]);
            }
          }
        }
      }
    } else {
      const bool odd = spin & 1;
#pragma unroll
      for (int cb = 0; cb < N; cb += 16) {
        // columns cb..cb+15 = 4 maps x (G re, G im, C re, C im)
        const float* p0 = acc + 0 * N + cb;  // F+, parity 0
        const float* p1 = acc + 1 * N + cb;  // F+, parity 1
        const float* m0 = acc + 2 * N + cb;  // F-, parity 0
        const float* m1 = acc + 3 * N + cb;  // F-, parity 1
        if (ring < Rh) {
#pragma unroll
          for (int q = 0; q < 16; q += 4) {
            const int bi = (cb + q) >> 2;
            if (b0 + bi >= B) continue;
            for (int side = 0; side < (rs != ring ? 2 : 1); ++side) {
              float gp_r, gp_i, cp_r, cp_i, gm_r, gm_i, cm_r, cm_i;
              if (side == 0) {
                gp_r = p0[q] + p1[q]; gp_i = p0[q + 1] + p1[q + 1];
                cp_r = p0[q + 2] + p1[q + 2]; cp_i = p0[q + 3] + p1[q + 3];
                gm_r = m0[q] + m1[q]; gm_i = m0[q + 1] + m1[q + 1];
                cm_r = m0[q + 2] + m1[q + 2]; cm_i = m0[q + 3] + m1[q + 3];
              } else {  // south: F+ -> p0 - p1, F- -> p1 - p0
                gp_r = p0[q] - p1[q]; gp_i = p0[q + 1] - p1[q + 1];
                cp_r = p0[q + 2] - p1[q + 2]; cp_i = p0[q + 3] - p1[q + 3];
                gm_r = m1[q] - m0[q]; gm_i = m1[q + 1] - m0[q + 1];
                cm_r = m1[q + 2] - m0[q + 2]; cm_i = m1[q + 3] - m0[q + 3];
              }
              float2 qv, uv;
              if (!odd) {  // Q = -(G F+ + i C F-), U = i G F- - C F+
                qv = make_float2(-(gp_r - cm_i), -(gp_i + cm_r));
                uv = make_float2(-gm_i - cp_r, gm_r - cp_i);
              } else {     // Q = -(G F- + i C F+), U = i G F+ - C F-
                qv = make_float2(-(gm_r - cp_i), -(gm_i + cp_r));
                uv = make_float2(-gp_i - cm_r, gp_r - cm_i);
              }
              const int rr = side == 0 ? ring : rs;
              const int64_t oo = ((int64_t(rr) * (mmax + 1) + m) * B + b0 + bi) * 2;
              phase[oo] = qv;
              phase[oo + 1] = uv;
            }
          }
        }
      }
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, NCOLS);
}

// ---------------------------------------------------------------- launchers
template <int NOPS, int BC>
static int launch_synth_tc(const Plan& P, const double2* almT, float2* phase, int B, int spin, int* err_flag,
                           cudaStream_t st) {
  using S = TcSmem<NOPS, 2 * NOPS * BC>;
  auto kern = synth_tc<NOPS, BC>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(S::DYN)) != cudaSuccess)
    return PS_ERR_CUDA;
  dim3 grid((P.Rh + TC_RT - 1) / TC_RT, P.mmax + 1, (B + BC - 1) / BC);
  kern<<<grid, TC_RT, S::DYN, st>>>(P.d_rings, P.d_mnorm0, spin ? P.d_seed[spin] : nullptr, almT, phase, P.R, P.Rh,
                                    P.lmax, P.mmax, B, spin, err_flag);
  PS_LAUNCH_CHECK();
  return PS_OK;
}

int launch_legendre_synth_tc(const Plan& P, const double2* almT, float2* phase, int B, int spin, int* err_flag,
                             cudaStream_t st) {
  const double flops = double(spin == 0 ? 4 : 16) * double(P.Rh) * double(P.nalm) * B;
  const double bytes = double(B) * (spin == 0 ? 1 : 2) * (16.0 * P.nalm + 8.0 * P.R * (P.mmax + 1));
  StatScope sc(PS_K_LEG_SYNTH, flops, bytes, st);
  // BC (maps per CTA): the plan's tile setting if any, else by batch size
  const int t = P.tile[0][spin];
  if (spin == 0) {
    const int bc = t ? t : (B > 16 ? 32 : B > 8 ? 16 : 8);
    if (bc == 32) return launch_synth_tc<1, 32>(P, almT, phase, B, 0, err_flag, st);
    if (bc == 16) return launch_synth_tc<1, 16>(P, almT, phase, B, 0, err_flag, st);
    return launch_synth_tc<1, 8>(P, almT, phase, B, 0, err_flag, st);
  }
  if (!P.d_seed[spin]) return PS_ERR_INVALID;
  const int bc = t ? t : (B > 4 ? 8 : 4);
  if (bc == 8) return launch_synth_tc<2, 8>(P, almT, phase, B, spin, err_flag, st);
  return launch_synth_tc<2, 4>(P, almT, phase, B, spin, err_flag, st);
}

}  // namespace ps
