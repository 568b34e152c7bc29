// Application of the masked-band ("cut") CG preconditioner in one C entry (ps_cutprec_apply):
//
//   M r = s + c,   s = Sigma r,
//   c   = Sigma B L^H Om^1/2 K_m^-1 Om^1/2 L B s     (per order m; m = 0 keeps Re c only)
//
// with L the Legendre synthesis stage on the masked band's rings (the band plan's table
// kernels, FP32 phases), Om^1/2 a per-(field, ring) weight and K_m^-1 the inverted band
// operator of order m (n = 3 R_b band coordinates: T rings, then Q rings, then U rings).
// The weighting of polyspec/weighting.py:76-78 (Sigma) and the CG operator of :297-299
// define the model; the Woodbury construction itself has no counterpart in the reference.
//
// Kernels, in order: Sigma r (ps_lm_matvec3, written straight into the output); a strided
// gather of B s into the Legendre stage's [nalm][batch][ncomp] layout; the band synthesis
// (spin 0, spin 2); cut_pack_y (phases times Om^1/2 -> the GEMM's B operand, BF16 in the
// tensor core's K-major core-matrix layout, `planes` = 1 (BF16) or 2 (BF16 hi + lo)); the
// per-m GEMM W_m = K_m^-1 Y_m (cut_gemm: tcgen05 kind::f16, K_m^-1 streamed from HBM by bulk
// copies straight into the MMA's operand layout, real and imaginary parts as two real
// MMAs into one accumulator: D = Re K [Yr | Yi] + Im K [-Yi | Yr] = [Re W | Im W]) whose
// epilogue writes Om^1/2 W back as band phases; the band adjoint writing B L^H (.) strided
// into a [batch][3][nalm] buffer; cut_finish adding Sigma of it (m = 0 real) to s.
#include <algorithm>
#include <cstring>

#include <cuda_bf16.h>

#include "ps_common.cuh"
#include "ps_stats.cuh"
#include "ps_tc.cuh"

struct ps_plan;

namespace ps {
int launch_tab_synth(const Plan& P, const float* table, const int64_t* d_blockoff, int Rh_table, int toff,
                     const double2* almT, float2* phase, int B, int spin, int* err_flag, cudaStream_t st, int fmt);
int launch_tab_adj(const Plan& P, const float* table, const int64_t* d_blockoff, const int2* d_work, int nwork,
                   int Rh_table, int toff, const float2* phase, double2* alm, int B, int spin, double scale,
                   int64_t out_stride, const double* lscale, int* err_flag, cudaStream_t st, int fmt);
// the band plan's Legendre tables (owned by its parent plan), resolved by the plan code
struct BandView {
  const Plan* P;
  const float* tab;
  const int64_t* off;
  const int2* work;
  int nwork, Rh_table, toff, fmt;
};
int band_view(const ps_plan* band, int spin, BandView& v);
}  // namespace ps

struct ps_cutprec {
  const ps_plan* plan;
  const ps_plan* band;
  int n, planes, M, RT, KS;  // band coordinates, BF16 planes, orders, row tiles, K stages
  int Rb;
  int64_t nalm;
  const double* om_half;  // [n]
  const double* sigma;    // [3][3][nalm]
  const double* beam;     // [3][nalm]
  uint16_t* kop;          // K_m^-1 in the GEMM layout, owned
  size_t kop_bytes;
};

namespace ps {
namespace {

constexpr int CUT_THREADS = 192;  // warp 0 copies, warp 1 MMA, warps 2..5 epilogue
constexpr uint32_t CUT_WAIT_LIMIT = 1u << 24;

size_t al256c(size_t x) { return (x + 255) & ~size_t(255); }

// element offset of (row, k) in a K-major no-swizzle tile of 16 K: 8 x 8 core matrices of 128 bytes,
// the two K halves adjacent, then the next 8-row group
__host__ __device__ __forceinline__ uint32_t kcore_el(int row, int k) {
  return uint32_t(((row >> 3) * 2 + (k >> 3)) * 64 + (row & 7) * 8 + (k & 7));
}
__device__ __forceinline__ uint64_t kdesc16(uint32_t saddr) {
  uint64_t d = 0;
  d |= uint64_t((saddr & 0x3FFFFu) >> 4);
  d |= uint64_t(128u >> 4) << 16;  // K-adjacent core matrices
  d |= uint64_t(256u >> 4) << 32;  // next 8-row group
  d |= uint64_t(1) << 46;
  return d;
}
__device__ __forceinline__ uint16_t bf16_rn(float x) {
  const __nv_bfloat16 h = __float2bfloat16_rn(x);
  return *reinterpret_cast<const uint16_t*>(&h);
}
__device__ __forceinline__ float bf16_val(uint16_t b) { return __uint_as_float(uint32_t(b) << 16); }

// ---- K_m^-1 (complex64 [M][n][n], row-major) -> [m][rt][ks][part][plane][128 x 16 BF16 tile]
__global__ void cut_kop_convert(const float2* __restrict__ kinv, int M, int n, int RT, int KS, int planes,
                                uint16_t* __restrict__ kop) {
  const int64_t per_m = int64_t(RT) * 128 * KS * 16;
  const int64_t total = int64_t(M) * per_m;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total; t += int64_t(gridDim.x) * blockDim.x) {
    const int m = int(t / per_m);
    int64_t rem = t - m * per_m;
    const int row = int(rem / (int64_t(KS) * 16));  // 0 .. RT*128
    const int col = int(rem - int64_t(row) * KS * 16);
    float2 v = make_float2(0.f, 0.f);
    if (row < n && col < n) v = kinv[(int64_t(m) * n + row) * n + col];
    const int rt = row >> 7, ks = col >> 4;
    const uint32_t el = kcore_el(row & 127, col & 15);
    const int64_t tile0 = ((int64_t(m) * RT + rt) * KS + ks) * 2 * planes;
#pragma unroll
    for (int part = 0; part < 2; ++part) {
      const float x = part ? v.y : v.x;
      const uint16_t hi = bf16_rn(x);
      kop[(tile0 + part * planes) * 2048 + el] = hi;
      if (planes == 2) kop[(tile0 + part * planes + 1) * 2048 + el] = bf16_rn(x - bf16_val(hi));
    }
  }
}

// ---- band phases (FP32, [Rb][M][Btot][nc], systems b0 .. b0 + B) times Om^1/2 -> the GEMM's B
// operand Yop [m][ks][variant][plane][N x 16], N = 2 Bp: variant 0 = [Yr | Yi], 1 = [-Yi | Yr]
__global__ void cut_pack_y(const float2* __restrict__ ph0, const float2* __restrict__ ph2,
                           const double* __restrict__ om_half, int Rb, int M, int Btot, int b0, int B, int Bp, int n,
                           int KS, int planes, uint16_t* __restrict__ yop) {
  const int N = 2 * Bp;
  const int64_t total = int64_t(M) * KS * 16 * Bp;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total; t += int64_t(gridDim.x) * blockDim.x) {
    const int b = int(t % Bp);
    const int64_t mj = t / Bp;
    const int j = int(mj % (int64_t(KS) * 16));
    const int m = int(mj / (int64_t(KS) * 16));
    float yr = 0.f, yi = 0.f;
    if (j < n && b < B) {
      const int f = j / Rb, r = j - f * Rb;
      const int64_t base = (int64_t(r) * M + m) * Btot + b0 + b;
      const float2 v = f == 0 ? ph0[base] : ph2[base * 2 + (f - 1)];
      const float w = float(om_half[j]);
      yr = v.x * w;
      yi = v.y * w;
    }
    const int ks = j >> 4, kk = j & 15;
    const int64_t tile0 = (int64_t(m) * KS + ks) * 2 * planes;  // [variant][plane] tiles of N x 16
    const float vals[2][2] = {{yr, yi}, {-yi, yr}};                // [variant][col half]
#pragma unroll
    for (int v = 0; v < 2; ++v)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const float x = vals[v][h];
        const uint32_t el = kcore_el(h * Bp + b, kk);
        const uint16_t hi = bf16_rn(x);
        yop[(tile0 + v * planes) * int64_t(N) * 16 + el] = hi;
        if (planes == 2) yop[(tile0 + v * planes + 1) * int64_t(N) * 16 + el] = bf16_rn(x - bf16_val(hi));
      }
  }
}

// bounded wait of one warp (lane 0 polls, the result is shared); the first to give up raises the
// CTA's abort flag and the plan's error flag
__device__ __forceinline__ bool cut_wait(uint32_t mbar, uint32_t parity, volatile int* abort, int* err_flag) {
  int ok = 1;
  if ((threadIdx.x & 31) == 0) {
    ok = 0;
    for (uint32_t i = 0; i < CUT_WAIT_LIMIT; ++i) {
      if (tc::mbar_try_wait(mbar, parity)) { ok = 1; break; }
      if ((i & 63) == 63 && *abort) break;
    }
    if (!ok && atomicExch(const_cast<int*>(abort), 1) == 0) atomicExch(err_flag, 1);
  }
  return __shfl_sync(0xffffffffu, ok, 0) != 0;
}

// One CTA = one row tile (128 band coordinates) of one order m, all systems of the chunk:
// D [128][N] = Sum_ks Re K(rt, ks) Y(ks, variant 0) + Im K(rt, ks) Y(ks, variant 1)  (P = 1), or the
// hi/lo products of both (P = 2: lo.hi and hi.lo first, hi.hi last).  Stage ks = 16 K values: the
// K tiles (2 P x 4 KB, contiguous in HBM for the CTA's whole row tile) and the Y tiles (2 P x N x 32 B,
// shared by the RT CTAs of the same m) land in a ring of NS stage buffers by bulk copies.
template <int P>
__global__ void __launch_bounds__(CUT_THREADS, 1) cut_gemm(const uint16_t* __restrict__ kop,
                                                           const uint16_t* __restrict__ yop, int M, int RT, int KS,
                                                           int n, int Rb, int Btot, int b0, int B, int Bp, int NS,
                                                           uint32_t tmem_cols, const double* __restrict__ om_half,
                                                           float2* __restrict__ ph0, float2* __restrict__ ph2,
                                                           int* __restrict__ err_flag) {
  extern __shared__ uint8_t cut_smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(cut_smem_raw) + 1023) & ~uintptr_t(1023));
  const int N = 2 * Bp;
  const uint32_t KST = 2u * P * 4096u;
  const uint32_t YST = 2u * P * uint32_t(N) * 32u;
  const uint32_t STG = KST + YST;
  const uint32_t sbase = tc::smem_u32(smem);
  const uint32_t misc = sbase + uint32_t(NS) * STG;
  const uint32_t full = misc, empty = misc + 64, done = misc + 128;
  volatile int* abort = reinterpret_cast<volatile int*>(smem + uint32_t(NS) * STG + 136);
  uint32_t* slot = reinterpret_cast<uint32_t*>(smem + uint32_t(NS) * STG + 144);
  const int rt = blockIdx.x % RT, m = blockIdx.x / RT;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp == 0) {
    tc::tmem_alloc(tc::smem_u32(slot), tmem_cols);
    tc::tmem_relinquish();
  }
  if (threadIdx.x == 0) {
    for (int i = 0; i < NS; ++i) {
      tc::mbar_init(full + 8u * uint32_t(i), 1);
      tc::mbar_init(empty + 8u * uint32_t(i), 1);
    }
    tc::mbar_init(done, 1);
    *abort = 0;
    tc::fence_mbar_init();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *slot;
  const uint16_t* ksrc = kop + (int64_t(m) * RT + rt) * KS * (2 * P * 2048);
  const uint16_t* ysrc = yop + int64_t(m) * KS * (2 * P * int64_t(N) * 16);

  if (warp == 0) {
    // ---- bulk copies of stage st into buffer st % NS
    int issued = 0;
    for (int st = 0; st < KS; ++st) {
      const int s = st % NS;
      if (st >= NS && !cut_wait(empty + 8u * uint32_t(s), uint32_t((st / NS) - 1) & 1u, abort, err_flag)) break;
      if (lane == 0) {
        const uint32_t bar = full + 8u * uint32_t(s);
        tc::mbar_arrive_expect_tx(bar, STG);
        tc::bulk_g2s(sbase + uint32_t(s) * STG, ksrc + int64_t(st) * (KST / 2), KST, bar);
        tc::bulk_g2s(sbase + uint32_t(s) * STG + KST, ysrc + int64_t(st) * (YST / 2), YST, bar);
      }
      __syncwarp();
      issued = st + 1;
    }
    // no copy may still be in flight when the CTA exits
    for (int st = max(0, issued - NS); st < issued; ++st) {
      int ok = 1;
      if (lane == 0) {
        ok = 0;
        for (uint32_t i = 0; i < CUT_WAIT_LIMIT; ++i)
          if (tc::mbar_try_wait(full + 8u * uint32_t(st % NS), uint32_t(st / NS) & 1u)) { ok = 1; break; }
        if (!ok) atomicExch(err_flag, 1);
      }
      __syncwarp();
      (void)ok;
    }
  } else if (warp == 1) {
    // ---- MMA issue
    const uint32_t idesc = tc::idesc_bf16(128, N, 0, 0);
    for (int st = 0; st < KS; ++st) {
      const int s = st % NS;
      if (!cut_wait(full + 8u * uint32_t(s), uint32_t(st / NS) & 1u, abort, err_flag)) break;
      tc::fence_after_sync();
      const uint32_t a0 = sbase + uint32_t(s) * STG, y0 = a0 + KST;
      const uint32_t ytile = uint32_t(N) * 32u;
      if (P == 1) {
        tc::mma_f16_elect(tmem, kdesc16(a0), kdesc16(y0), idesc, st > 0 ? 1u : 0u);
        tc::mma_f16_elect(tmem, kdesc16(a0 + 4096u), kdesc16(y0 + ytile), idesc, 1u);
      } else {
        // tiles: K [part][plane], Y [variant][plane]; plane 0 = hi, 1 = lo
        const uint32_t kre_h = a0, kre_l = a0 + 4096u, kim_h = a0 + 8192u, kim_l = a0 + 12288u;
        const uint32_t y0_h = y0, y0_l = y0 + ytile, y1_h = y0 + 2 * ytile, y1_l = y0 + 3 * ytile;
        tc::mma_f16_elect(tmem, kdesc16(kre_l), kdesc16(y0_h), idesc, st > 0 ? 1u : 0u);
        tc::mma_f16_elect(tmem, kdesc16(kre_h), kdesc16(y0_l), idesc, 1u);
        tc::mma_f16_elect(tmem, kdesc16(kim_l), kdesc16(y1_h), idesc, 1u);
        tc::mma_f16_elect(tmem, kdesc16(kim_h), kdesc16(y1_l), idesc, 1u);
        tc::mma_f16_elect(tmem, kdesc16(kre_h), kdesc16(y0_h), idesc, 1u);
        tc::mma_f16_elect(tmem, kdesc16(kim_h), kdesc16(y1_h), idesc, 1u);
      }
      tc::mma_commit_elect(empty + 8u * uint32_t(s));
    }
    tc::mma_commit_elect(done);
  } else {
    // ---- epilogue: warp w reads TMEM lane quarter w & 3; row = band coordinate rt * 128 + row
    const int q = warp & 3;
    const bool ok = cut_wait(done, 0u, abort, err_flag);
    tc::fence_after_sync();
    const int row = 32 * q + lane;
    const int i = rt * 128 + row;
    const uint32_t lane_addr = tmem + (uint32_t(32 * q) << 16);
    const bool live = ok && !*abort && i < n;
    int f = 0, r = 0;
    float w = 0.f;
    if (i < n) {
      f = i / Rb;
      r = i - f * Rb;
      w = float(om_half[i]);
    }
    for (int c0 = 0; c0 < Bp; c0 += 16) {
      float re[16], im[16];
      tc::tmem_ld16(lane_addr + uint32_t(c0), re);
      tc::tmem_ld16(lane_addr + uint32_t(Bp + c0), im);
      tc::tmem_ld_wait();
      if (live) {
#pragma unroll
        for (int k = 0; k < 16; ++k) {
          const int b = c0 + k;
          if (b < B) {
            const int64_t idx = (int64_t(r) * M + m) * Btot + b0 + b;
            const float2 v = make_float2(re[k] * w, im[k] * w);
            if (f == 0)
              ph0[idx] = v;
            else
              ph2[idx * 2 + (f - 1)] = v;
          }
        }
      }
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, tmem_cols);
}

// B s -> almT [nalm][B][ncomp] for components c0 .. c0 + ncomp of x [B][3][nalm]
__global__ void cut_gather(const double2* __restrict__ x, const double* __restrict__ beam, int c0, int ncomp,
                           double2* __restrict__ almT, int B, int64_t nalm) {
  const int64_t total = nalm * B * ncomp;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total; t += int64_t(gridDim.x) * blockDim.x) {
    const int c = int(t % ncomp);
    const int b = int((t / ncomp) % B);
    const int64_t idx = t / (int64_t(ncomp) * B);
    const double2 v = x[(int64_t(b) * 3 + c0 + c) * nalm + idx];
    almT[t] = cscale(v, beam[int64_t(c0 + c) * nalm + idx]);
  }
}

// out[b][a][i] += Sum_c Sigma[a][c][i] a[b][c][i], with the imaginary part of the sum dropped at m = 0
// (alm index i <= lmax)
__global__ void cut_finish(const double* __restrict__ S, const double2* __restrict__ a, double2* __restrict__ out,
                           int B, int64_t nalm, int lmax) {
  const int64_t total = int64_t(B) * nalm;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total; t += int64_t(gridDim.x) * blockDim.x) {
    const int64_t b = t / nalm, i = t - b * nalm;
    double2 v[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) v[c] = a[(b * 3 + c) * nalm + i];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      double2 s = make_double2(0.0, 0.0);
#pragma unroll
      for (int c = 0; c < 3; ++c) s = cfma(__ldg(S + (int64_t(r) * 3 + c) * nalm + i), v[c], s);
      if (i <= lmax) s.y = 0.0;
      double2& o = out[(b * 3 + r) * nalm + i];
      o = cadd(o, s);
    }
  }
}

int cut_grid(int64_t n) {
  const int64_t need = (n + 255) / 256, cap = int64_t(device_sms()) * 8;
  return int(std::max<int64_t>(1, std::min(need, cap)));
}

int cut_bp(int B) { return (B + 15) & ~15; }
constexpr int CUT_BMAX = 128;  // systems per GEMM pass (N = 2 Bp <= 256)

struct CutLayout {
  size_t almT, ph0, ph2, yop, a, total;
};
CutLayout cut_layout(const ps_cutprec* c, int B) {
  CutLayout L;
  size_t o = 0;
  const int Bc = std::min(B, CUT_BMAX);
  L.almT = o; o += al256c(size_t(c->nalm) * B * 2 * sizeof(double2));
  L.ph0 = o; o += al256c(size_t(c->Rb) * c->M * B * sizeof(float2));
  L.ph2 = o; o += al256c(size_t(c->Rb) * c->M * B * 2 * sizeof(float2));
  L.yop = o; o += al256c(size_t(c->M) * c->KS * 2 * c->planes * size_t(2 * cut_bp(Bc)) * 16 * sizeof(uint16_t));
  L.a = o; o += al256c(size_t(B) * 3 * c->nalm * sizeof(double2));
  L.total = o;
  return L;
}

template <int P>
int launch_cut_gemm(const ps_cutprec* c, const uint16_t* yop, int Btot, int b0, int B, float2* ph0, float2* ph2,
                    int* err, cudaStream_t st) {
  const int Bp = cut_bp(B), N = 2 * Bp;
  const uint32_t STG = 2u * P * 4096u + 2u * P * uint32_t(N) * 32u;
  const int NS = int(std::max<uint32_t>(2u, std::min<uint32_t>(8u, (100u * 1024u) / STG)));
  const size_t smem = 1024 + size_t(NS) * STG + 256;
  uint32_t cols = 32;
  while (cols < uint32_t(N)) cols <<= 1;
  static bool attr = false;
  if (!attr) {
    if (cudaFuncSetAttribute(cut_gemm<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024) != cudaSuccess)
      return PS_ERR_CUDA;
    attr = true;
  }
  // algorithmic bytes: K_m^-1 once, the B operand once, the output phases
  StatScope sc(PS_K_VECTOR, 8.0 * double(c->M) * c->n * c->n * B * (P == 1 ? 1 : 3),
               double(c->kop_bytes) + double(c->M) * c->KS * 2 * P * N * 32 + 8.0 * double(c->n) * c->M * B, st);
  cut_gemm<P><<<c->M * c->RT, CUT_THREADS, smem, st>>>(c->kop, yop, c->M, c->RT, c->KS, c->n, c->Rb, Btot, b0, B,
                                                      Bp, NS, cols, c->om_half, ph0, ph2, err);
  PS_LAUNCH_CHECK();
  return PS_OK;
}

}  // namespace
}  // namespace ps

using namespace ps;

extern "C" int ps_cutprec_create(const ps_plan* plan, const ps_plan* band, const void* kinv, int n, int planes,
                                 const double* om_half, const double* sigma, const double* beam, cudaStream_t stream,
                                 ps_cutprec** out) {
  if (!out) return PS_ERR_INVALID;
  *out = nullptr;
  if (!plan || !band || !kinv || !om_half || !sigma || !beam || n <= 0 || (planes != 1 && planes != 2))
    return PS_ERR_INVALID;
  BandView v0, v2;
  int rc = band_view(band, 0, v0);
  if (rc == PS_OK) rc = band_view(band, 2, v2);
  if (rc != PS_OK) return rc;
  int lmax = 0;
  int64_t nalm = 0;
  rc = ps_plan_info(plan, nullptr, &lmax, nullptr, &nalm);
  if (rc != PS_OK) return rc;
  const Plan& B = *v0.P;
  if (B.nalm != nalm || 3 * B.R != n) return PS_ERR_INVALID;
  ps_cutprec* c = new ps_cutprec();
  c->plan = plan;
  c->band = band;
  c->n = n;
  c->planes = planes;
  c->M = B.mmax + 1;
  c->RT = (n + 127) / 128;
  c->KS = (n + 15) / 16;
  c->Rb = B.R;
  c->nalm = nalm;
  c->om_half = om_half;
  c->sigma = sigma;
  c->beam = beam;
  c->kop_bytes = size_t(c->M) * c->RT * c->KS * 2 * planes * 4096;
  if (cudaMalloc(&c->kop, c->kop_bytes) != cudaSuccess) {
    cudaGetLastError();
    delete c;
    return PS_ERR_NOMEM;
  }
  const int64_t total = int64_t(c->M) * c->RT * 128 * c->KS * 16;
  cut_kop_convert<<<cut_grid(total), 256, 0, stream>>>(static_cast<const float2*>(kinv), c->M, n, c->RT, c->KS,
                                                       planes, c->kop);
  if (cudaGetLastError() != cudaSuccess) {
    cudaFree(c->kop);
    delete c;
    return PS_ERR_CUDA;
  }
  *out = c;
  return PS_OK;
}

extern "C" int ps_cutprec_destroy(ps_cutprec* c) {
  if (!c) return PS_ERR_INVALID;
  cudaFree(c->kop);
  delete c;
  return PS_OK;
}

extern "C" int ps_cutprec_workspace_bytes(const ps_cutprec* c, int batch, size_t* bytes) {
  if (!c || !bytes || batch <= 0) return PS_ERR_INVALID;
  *bytes = cut_layout(c, batch).total;
  return PS_OK;
}

extern "C" int ps_cutprec_apply(const ps_cutprec* c, const double* r, double* out, int batch, void* workspace,
                                size_t workspace_bytes, cudaStream_t stream) {
  if (!c || !r || !out || batch < 0 || r == out) return PS_ERR_INVALID;
  if (batch == 0) return PS_OK;
  const CutLayout L = cut_layout(c, batch);
  if (!workspace || workspace_bytes < L.total) return PS_ERR_WORKSPACE;
  BandView v0, v2;
  int rc = band_view(c->band, 0, v0);
  if (rc == PS_OK) rc = band_view(c->band, 2, v2);
  if (rc != PS_OK) return rc;
  char* ws = static_cast<char*>(workspace);
  double2* almT = reinterpret_cast<double2*>(ws + L.almT);
  float2* ph0 = reinterpret_cast<float2*>(ws + L.ph0);
  float2* ph2 = reinterpret_cast<float2*>(ws + L.ph2);
  uint16_t* yop = reinterpret_cast<uint16_t*>(ws + L.yop);
  double2* a = reinterpret_cast<double2*>(ws + L.a);
  double2* o = reinterpret_cast<double2*>(out);
  const int64_t nalm = c->nalm;
  int* err = v0.P->d_err;
  // s = Sigma r, straight into the output
  rc = ps_lm_matvec3(c->sigma, nullptr, nullptr, r, out, batch, nalm, stream);
  if (rc != PS_OK) return rc;
  // band synthesis of B s, spin 0 (T) then spin 2 (E, B)
  for (int spin = 0; spin <= 2; spin += 2) {
    const int nc = spin ? 2 : 1;
    const BandView& v = spin ? v2 : v0;
    {
      StatScope sc(PS_K_LAYOUT, 0.0, 40.0 * double(nalm) * batch * nc, stream);
      cut_gather<<<cut_grid(nalm * batch * nc), 256, 0, stream>>>(o, c->beam, spin ? 1 : 0, nc, almT, batch, nalm);
      PS_LAUNCH_CHECK();
    }
    rc = launch_tab_synth(*v.P, v.tab, v.off, v.Rh_table, v.toff, almT, spin ? ph2 : ph0, batch, spin, err, stream,
                          v.fmt);
    if (rc != PS_OK) return rc;
  }
  // W = K_m^-1 Y per order, at most CUT_BMAX systems per pass, written back over the phases
  for (int b0 = 0; b0 < batch; b0 += CUT_BMAX) {
    const int B = std::min(CUT_BMAX, batch - b0), Bp = cut_bp(B);
    {
      const int64_t total = int64_t(c->M) * c->KS * 16 * Bp;
      StatScope sc(PS_K_LAYOUT, 0.0, 8.0 * double(c->n) * c->M * B + 2.0 * c->planes * 4.0 * double(total), stream);
      cut_pack_y<<<cut_grid(total), 256, 0, stream>>>(ph0, ph2, c->om_half, c->Rb, c->M, batch, b0, B, Bp, c->n,
                                                      c->KS, c->planes, yop);
      PS_LAUNCH_CHECK();
    }
    rc = c->planes == 1 ? launch_cut_gemm<1>(c, yop, batch, b0, B, ph0, ph2, err, stream)
                        : launch_cut_gemm<2>(c, yop, batch, b0, B, ph0, ph2, err, stream);
    if (rc != PS_OK) return rc;
  }
  // band adjoint with the beam, strided into a [batch][3][nalm]
  for (int spin = 0; spin <= 2; spin += 2) {
    const BandView& v = spin ? v2 : v0;
    const int c0 = spin ? 1 : 0;
    rc = launch_tab_adj(*v.P, v.tab, v.off, v.work, v.nwork, v.Rh_table, v.toff, spin ? ph2 : ph0, a + c0 * nalm,
                        batch, spin, 1.0, 3 * nalm, c->beam + c0 * nalm, err, stream, v.fmt);
    if (rc != PS_OK) return rc;
  }
  int lmax = 0;
  ps_plan_info(c->plan, nullptr, &lmax, nullptr, nullptr);
  StatScope sc(PS_K_VECTOR, 36.0 * batch * double(nalm), 168.0 * batch * double(nalm) + 72.0 * nalm, stream);
  cut_finish<<<cut_grid(int64_t(batch) * nalm), 256, 0, stream>>>(c->sigma, a, o, batch, nalm, lmax);
  PS_LAUNCH_CHECK();
  return PS_OK;
}
