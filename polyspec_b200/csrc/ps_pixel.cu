// Pixel-space products, radial sums and harmonic weightings of the
// TSpecTemplate / ideal-Fisher path (FP64, HBM-bound).
//
//  * ps_pix_product: the elementwise map products of polyspec/cython/
//    tauNL_utils.pyx:103-215 and ideal_fisher.pyx:18-157 (one templated
//    grid-stride kernel per product; every input and the output are streamed
//    once, 8-byte real or 16-byte complex words per thread, coalesced).
//  * ps_pix_radial_sum: the quartic pixel sums Sum_r w_r Sum_pix f(maps)
//    of tauNL_utils.pyx:260-405.  Stage 1: grid (chunks, rings) of CTAs, each
//    reduces a contiguous chunk of one radial sample's maps (warp shuffles,
//    then one value per warp in shared memory) into partial[r][chunk].
//    Stage 2: one CTA adds the partials in a fixed order, times the radial
//    weights, in FP64 -- the result does not depend on scheduling.
//  * ps_apply_fl_weights / ps_radial_sum_lm: the harmonic weightings
//    tauNL_utils.pyx:80-98 and :220-255 (thread per lm, radial samples looped
//    in registers; f_l^X(r) gathered by l from L2).
//  * ps_outer_product: the Fisher outer product ideal_fisher.pyx:423-460
//    (split over j in chunks; 16 x 16 (a, b) tile per CTA with Q tiles staged
//    in shared memory; partials added in a fixed order by a second kernel).
#include "ps_common.cuh"
#include "ps_stats.cuh"

namespace ps {
namespace {

constexpr int PIX_THREADS = 256;

struct PixIn {
  const void* p[8];
  void* out;
  int64_t n;
  int npol;
  double fac;
};

__device__ __forceinline__ double ldr(const void* p, int64_t i) {
  return __ldg(static_cast<const double*>(p) + i);
}
__device__ __forceinline__ double2 ldc(const void* p, int64_t i) {
  return __ldg(static_cast<const double2*>(p) + i);
}
__device__ __forceinline__ double re_conj_mul(double2 a, double2 b) {  // Re(a conj(b)) = Re(conj(a) b)
  return a.x * b.x + a.y * b.y;
}
__device__ __forceinline__ double2 cmul_conj(double2 a, double2 b) {  // a * conj(b)
  return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ double2 conj_mul(double2 a, double2 b) {  // conj(a) * b
  return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}

// one element of each product; the expressions follow the reference's,
// term by term (tauNL_utils.pyx / ideal_fisher.pyx line ranges beside each op)
template <int OP>
__device__ __forceinline__ void pix_elem(const PixIn& a, int64_t i) {
  if constexpr (OP == PS_PIX_MULTIPLY) {  // tauNL_utils.pyx:103-113  m1 m2 m3
    static_cast<double*>(a.out)[i] = ldr(a.p[0], i) * ldr(a.p[1], i) * ldr(a.p[2], i);
  } else if constexpr (OP == PS_PIX_MULTIPLY_ASYM) {  // :116-126  m1A (2 m1B m3A + m1A m3B)
    const double m1a = ldr(a.p[0], i);
    static_cast<double*>(a.out)[i] = m1a * (2 * ldr(a.p[1], i) * ldr(a.p[2], i) + m1a * ldr(a.p[3], i));
  } else if constexpr (OP == PS_PIX_MULTIPLYC) {  // :129-139  m1 m2 m3c
    const double s = ldr(a.p[0], i) * ldr(a.p[1], i);
    const double2 c = ldc(a.p[2], i);
    static_cast<double2*>(a.out)[i] = make_double2(s * c.x, s * c.y);
  } else if constexpr (OP == PS_PIX_MULTIPLYC_ASYM) {  // :142-152  m1A (2 m1B cA + m1A cB)
    const double m1a = ldr(a.p[0], i), m1b = ldr(a.p[1], i);
    const double2 ca = ldc(a.p[2], i), cb = ldc(a.p[3], i);
    static_cast<double2*>(a.out)[i] =
        make_double2(m1a * (2 * m1b * ca.x + m1a * cb.x), m1a * (2 * m1b * ca.y + m1a * cb.y));
  } else if constexpr (OP == PS_PIX_MULTIPLYCC) {  // :155-165  m1 (m2^2 + |c|^2)
    const double m2 = ldr(a.p[1], i);
    const double2 c = ldc(a.p[2], i);
    static_cast<double*>(a.out)[i] = ldr(a.p[0], i) * (m2 * m2 + (c.x * c.x + c.y * c.y));
  } else if constexpr (OP == PS_PIX_MULTIPLYCC_ASYM) {
    // :168-178  2 m1A (m2A m2B + Re(conj(cA) cB)) + m1B (m2A^2 + |cA|^2)
    const double m1a = ldr(a.p[0], i), m1b = ldr(a.p[1], i), m2a = ldr(a.p[2], i), m2b = ldr(a.p[3], i);
    const double2 ca = ldc(a.p[4], i), cb = ldc(a.p[5], i);
    static_cast<double*>(a.out)[i] =
        2 * m1a * (m2a * m2b + re_conj_mul(ca, cb)) + m1b * (m2a * m2a + (ca.x * ca.x + ca.y * ca.y));
  } else if constexpr (OP == PS_PIX_MULTIPLY2) {  // :181-191  B1 B2 + Re(C1 conj(C2))
    static_cast<double*>(a.out)[i] = ldr(a.p[0], i) * ldr(a.p[1], i) + re_conj_mul(ldc(a.p[2], i), ldc(a.p[3], i));
  } else if constexpr (OP == PS_PIX_MULTIPLY2R || OP == PS_PIX_MULTIPLYRR) {
    // tauNL_utils.pyx:194-204, ideal_fisher.pyx:100-108  A B
    static_cast<double*>(a.out)[i] = ldr(a.p[0], i) * ldr(a.p[1], i);
  } else if constexpr (OP == PS_PIX_MULTIPLY2C) {  // tauNL_utils.pyx:207-217  Ac B
    const double2 c = ldc(a.p[0], i);
    const double b = ldr(a.p[1], i);
    static_cast<double2*>(a.out)[i] = make_double2(c.x * b, c.y * b);
  } else if constexpr (OP == PS_PIX_MULTIPLYRC) {  // ideal_fisher.pyx:52-60  R C
    const double r = ldr(a.p[0], i);
    const double2 c = ldc(a.p[1], i);
    static_cast<double2*>(a.out)[i] = make_double2(r * c.x, r * c.y);
  } else if constexpr (OP == PS_PIX_MULTIPLYRCSTAR) {  // :64-72  fac R conj(C)
    const double r = ldr(a.p[0], i);
    const double2 c = ldc(a.p[1], i);
    static_cast<double2*>(a.out)[i] = make_double2(a.fac * r * c.x, -(a.fac * r * c.y));
  } else if constexpr (OP == PS_PIX_MULTIPLYRC_SYM) {  // :76-84  R C + R2 C2
    const double r = ldr(a.p[0], i), r2 = ldr(a.p[2], i);
    const double2 c = ldc(a.p[1], i), c2 = ldc(a.p[3], i);
    static_cast<double2*>(a.out)[i] = make_double2(r * c.x + r2 * c2.x, r * c.y + r2 * c2.y);
  } else if constexpr (OP == PS_PIX_MULTIPLYRCSTAR_SYM) {  // :88-96  fac (R conj(C) + R2 conj(C2))
    const double r = ldr(a.p[0], i), r2 = ldr(a.p[2], i);
    const double2 c = ldc(a.p[1], i), c2 = ldc(a.p[3], i);
    static_cast<double2*>(a.out)[i] =
        make_double2(a.fac * (r * c.x + r2 * c2.x), a.fac * (-(r * c.y) - r2 * c2.y));
  } else if constexpr (OP == PS_PIX_MULTIPLYRR_SYM) {  // :112-120  A B + A' B'
    static_cast<double*>(a.out)[i] = ldr(a.p[0], i) * ldr(a.p[1], i) + ldr(a.p[2], i) * ldr(a.p[3], i);
  } else if constexpr (OP == PS_PIX_R2C) {  // :18-26  re + i im
    static_cast<double2*>(a.out)[i] = make_double2(ldr(a.p[0], i), ldr(a.p[1], i));
  } else if constexpr (OP == PS_PIX_R2CSTAR) {  // :30-38  re - i im
    static_cast<double2*>(a.out)[i] = make_double2(ldr(a.p[0], i), -ldr(a.p[1], i));
  } else if constexpr (OP == PS_PIX_PRODUCT_REAL1) {  // ideal_fisher.pyx:177-190, :325-338 (one term)  fac A B
    static_cast<double*>(a.out)[i] = a.fac * ldr(a.p[0], i) * ldr(a.p[1], i);
  } else if constexpr (OP == PS_PIX_PRODUCT_REAL2) {  // the same with two terms  fac A0 B0 + fac A1 B1
    static_cast<double*>(a.out)[i] =
        a.fac * ldr(a.p[0], i) * ldr(a.p[1], i) + a.fac * ldr(a.p[2], i) * ldr(a.p[3], i);
  } else if constexpr (OP == PS_PIX_LENS_PHI || OP == PS_PIX_LENS_PHI_SYM) {
    // ideal_fisher.pyx:124-157.  Spin 0: 2 U0 conj(V0).  With polarisation:
    //   2 U0 conj(V0) + (U1 conj(V1) - conj(U1) V2) + i (U2 conj(V1) + conj(U2) V2)
    // and the symmetrised form adds the same with (U, V) = (U2, V1).
    const int64_t n = a.n;
    auto one = [&](const void* U, const void* V) {
      const double2 u0 = ldc(U, i), v0 = ldc(V, i);
      double2 t = cmul_conj(u0, v0);
      t.x *= 2; t.y *= 2;
      if (a.npol == 3) {
        const double2 u1 = ldc(U, n + i), u2 = ldc(U, 2 * n + i), v1 = ldc(V, n + i), v2 = ldc(V, 2 * n + i);
        const double2 p = cmul_conj(u1, v1), q = conj_mul(u1, v2);
        const double2 r = cmul_conj(u2, v1), s = conj_mul(u2, v2);
        const double2 w = make_double2(r.x + s.x, r.y + s.y);  // times i
        t.x += (p.x - q.x) - w.y;
        t.y += (p.y - q.y) + w.x;
      }
      return t;
    };
    if constexpr (OP == PS_PIX_LENS_PHI) {
      static_cast<double2*>(a.out)[i] = one(a.p[0], a.p[1]);
    } else {  // inputs U1, U2, V1, V2:  f(U1, V2) + f(U2, V1)
      const double2 t1 = one(a.p[0], a.p[3]), t2 = one(a.p[1], a.p[2]);
      static_cast<double2*>(a.out)[i] = make_double2(t1.x + t2.x, t1.y + t2.y);
    }
  }
}

template <int OP>
__global__ void __launch_bounds__(PIX_THREADS) pix_product_kernel(PixIn a) {
  const int64_t stride = int64_t(gridDim.x) * PIX_THREADS;
  int64_t i = int64_t(blockIdx.x) * PIX_THREADS + threadIdx.x;
  // two elements per iteration: both loads are in flight before either store
  for (; i + stride < a.n; i += 2 * stride) {
    pix_elem<OP>(a, i);
    pix_elem<OP>(a, i + stride);
  }
  if (i < a.n) pix_elem<OP>(a, i);
}

struct OpInfo {
  int n_in;
  double bytes_per_elem;  // algorithmic bytes moved per output element
};

OpInfo op_info(int op, int npol) {
  switch (op) {
    case PS_PIX_MULTIPLY: return {3, 32};
    case PS_PIX_MULTIPLY_ASYM: return {4, 40};
    case PS_PIX_MULTIPLYC: return {3, 48};
    case PS_PIX_MULTIPLYC_ASYM: return {4, 64};
    case PS_PIX_MULTIPLYCC: return {3, 40};
    case PS_PIX_MULTIPLYCC_ASYM: return {6, 72};
    case PS_PIX_MULTIPLY2: return {4, 56};
    case PS_PIX_MULTIPLY2R: return {2, 24};
    case PS_PIX_MULTIPLY2C: return {2, 40};
    case PS_PIX_MULTIPLYRC: return {2, 40};
    case PS_PIX_MULTIPLYRCSTAR: return {2, 40};
    case PS_PIX_MULTIPLYRC_SYM: return {4, 64};
    case PS_PIX_MULTIPLYRCSTAR_SYM: return {4, 64};
    case PS_PIX_MULTIPLYRR: return {2, 24};
    case PS_PIX_MULTIPLYRR_SYM: return {4, 40};
    case PS_PIX_R2C: return {2, 32};
    case PS_PIX_R2CSTAR: return {2, 32};
    case PS_PIX_LENS_PHI: return {2, 16.0 + 32.0 * npol};
    case PS_PIX_LENS_PHI_SYM: return {4, 16.0 + 64.0 * npol};
    case PS_PIX_PRODUCT_REAL1: return {2, 24};
    case PS_PIX_PRODUCT_REAL2: return {4, 40};
    default: return {-1, 0};
  }
}

int grid_for(int64_t n, int sms) {
  // enough resident CTAs to cover HBM latency (8 per SM x 256 threads), a multiple of the SM count
  const int64_t need = (n + PIX_THREADS - 1) / PIX_THREADS;
  const int64_t cap = int64_t(sms) * 8;
  return int(need < cap ? need : cap);
}

int g_sms = 0;
int sm_count() {
  if (g_sms == 0) {
    int dev = 0, c = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, dev);
    g_sms = c > 0 ? c : 148;
  }
  return g_sms;
}

template <int OP>
void launch_op(const PixIn& a, int grid, cudaStream_t st) {
  pix_product_kernel<OP><<<grid, PIX_THREADS, 0, st>>>(a);
}

// ------------------------------------------------------------------ radial sums
constexpr int SUM_THREADS = 256;
constexpr int SUM_MAX_CHUNKS = 64;

struct SumIn {
  const void* p[8];
  int64_t npix;
  int nchunks;
};

template <int KIND>
__device__ __forceinline__ double sum_term(const SumIn& a, int64_t o) {
  // o = r * npix + pixel.  Terms follow tauNL_utils.pyx:260-405.
  if constexpr (KIND == PS_SUM_GNL_LOC) {  // P^3 Q
    const double p = ldr(a.p[0], o);
    return p * p * p * ldr(a.p[1], o);
  } else if constexpr (KIND == PS_SUM_GNL_LOC_DISC) {  // P1^2 P2 Q2 + P2^2 P1 Q1
    const double p1 = ldr(a.p[0], o), p2 = ldr(a.p[1], o);
    return p1 * p1 * p2 * ldr(a.p[3], o) + p2 * p2 * p1 * ldr(a.p[2], o);
  } else if constexpr (KIND == PS_SUM_GNL_CON || KIND == PS_SUM_GNL_DOTDOT) {  // R^4
    const double r = ldr(a.p[0], o);
    const double r2 = r * r;
    return r2 * r2;
  } else if constexpr (KIND == PS_SUM_GNL_CON_DISC || KIND == PS_SUM_GNL_DOTDOT_DISC) {  // R1^2 R2^2
    const double r1 = ldr(a.p[0], o), r2 = ldr(a.p[1], o);
    return r1 * r1 * (r2 * r2);
  } else if constexpr (KIND == PS_SUM_GNL_DOTDEL) {  // A^2 (B^2 + |C|^2)
    const double A = ldr(a.p[0], o), B = ldr(a.p[1], o);
    const double2 C = ldc(a.p[2], o);
    return A * A * (B * B + (C.x * C.x + C.y * C.y));
  } else if constexpr (KIND == PS_SUM_GNL_DOTDEL_DISC) {  // A1 A2 (B1 B2 + Re(C1 conj C2))
    const double2 c1 = ldc(a.p[4], o), c2 = ldc(a.p[5], o);
    return ldr(a.p[0], o) * ldr(a.p[1], o) * (ldr(a.p[2], o) * ldr(a.p[3], o) + re_conj_mul(c1, c2));
  } else if constexpr (KIND == PS_SUM_GNL_DELDEL) {  // (B^2 + |C|^2)^2
    const double B = ldr(a.p[0], o);
    const double2 C = ldc(a.p[1], o);
    const double t = B * B + (C.x * C.x + C.y * C.y);
    return t * t;
  } else {  // PS_SUM_GNL_DELDEL_DISC: (B1 B2 + Re(C1 conj C2)) (B3 B4 + Re(C3 conj C4))
    const double t1 = ldr(a.p[0], o) * ldr(a.p[1], o) + re_conj_mul(ldc(a.p[4], o), ldc(a.p[5], o));
    const double t2 = ldr(a.p[2], o) * ldr(a.p[3], o) + re_conj_mul(ldc(a.p[6], o), ldc(a.p[7], o));
    return t1 * t2;
  }
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

template <int KIND>
__global__ void __launch_bounds__(SUM_THREADS) radial_sum_stage1(SumIn a, double* __restrict__ partial) {
  const int r = blockIdx.y, c = blockIdx.x;
  const int64_t per = (a.npix + a.nchunks - 1) / a.nchunks;
  const int64_t lo = int64_t(c) * per, hi = min(a.npix, lo + per);
  const int64_t base = int64_t(r) * a.npix;
  double s0 = 0.0, s1 = 0.0;
  int64_t i = lo + threadIdx.x;
  for (; i + SUM_THREADS < hi; i += 2 * SUM_THREADS) {
    s0 += sum_term<KIND>(a, base + i);
    s1 += sum_term<KIND>(a, base + i + SUM_THREADS);
  }
  if (i < hi) s0 += sum_term<KIND>(a, base + i);
  double v = warp_sum(s0 + s1);
  __shared__ double sw[SUM_THREADS / 32];
  if ((threadIdx.x & 31) == 0) sw[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < SUM_THREADS / 32; ++w) t += sw[w];
    partial[int64_t(r) * a.nchunks + c] = t;
  }
}

// out = Sum_r weight_r * Sum_c partial[r][c], weight_r = w_r tau_r^tpow (fixed order)
__global__ void radial_sum_stage2(const double* __restrict__ partial, const double* __restrict__ w,
                                  const double* __restrict__ tau, int tpow, int nr, int nchunks,
                                  double* __restrict__ out) {
  __shared__ double s[256];
  double acc = 0.0;
  for (int r = threadIdx.x; r < nr; r += blockDim.x) {
    double t = 0.0;
    for (int c = 0; c < nchunks; ++c) t += partial[int64_t(r) * nchunks + c];
    double wr = w[r];
    if (tpow > 0) {
      const double t2 = tau[r] * tau[r];
      wr *= (tpow == 4) ? t2 * t2 : t2;
    }
    acc += wr * t;
  }
  s[threadIdx.x] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int k = 0; k < int(blockDim.x); ++k) t += s[k];
    *out = t;
  }
}

struct SumInfo {
  int n_maps;
  int tpow;          // power of tau in the radial weight
  double bytes_pix;  // algorithmic bytes per (r, pixel)
};

SumInfo sum_info(int kind) {
  switch (kind) {
    case PS_SUM_GNL_LOC: return {2, 0, 16};
    case PS_SUM_GNL_LOC_DISC: return {4, 0, 32};
    case PS_SUM_GNL_CON: return {1, 0, 8};
    case PS_SUM_GNL_CON_DISC: return {2, 0, 16};
    case PS_SUM_GNL_DOTDOT: return {1, 4, 8};
    case PS_SUM_GNL_DOTDOT_DISC: return {2, 4, 16};
    case PS_SUM_GNL_DOTDEL: return {3, 2, 32};
    case PS_SUM_GNL_DOTDEL_DISC: return {6, 2, 64};
    case PS_SUM_GNL_DELDEL: return {2, 0, 24};
    case PS_SUM_GNL_DELDEL_DISC: return {8, 0, 96};
    default: return {-1, 0, 0};
  }
}

int sum_chunks(int nr, int64_t npix) {
  // about 4 CTAs per SM over all radial samples, at least 16 K pixels per CTA
  int c = int((int64_t(sm_count()) * 4 + nr - 1) / nr);
  const int64_t maxc = (npix + 16383) / 16384;
  if (c > maxc) c = int(maxc);
  if (c > SUM_MAX_CHUNKS) c = SUM_MAX_CHUNKS;
  return c < 1 ? 1 : c;
}

template <int KIND>
void launch_sum(const SumIn& a, int nr, double* partial, cudaStream_t st) {
  dim3 grid(a.nchunks, nr);
  radial_sum_stage1<KIND><<<grid, SUM_THREADS, 0, st>>>(a, partial);
}

// ------------------------------------------------------------------ harmonic weightings
// out[r][lm] = weight * Sum_X flX[l][X][r] h[X][lm]        (tauNL_utils.pyx:80-98)
// (an l outside [0, lsize) gives zeros instead of reading past flX)
__global__ void apply_fl_kernel(const double* __restrict__ flX, int lsize, int npol, int nr,
                                const double2* __restrict__ h, const int* __restrict__ ls, int64_t nlm, double weight,
                                double2* __restrict__ out) {
  const int64_t ilm = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (ilm >= nlm) return;
  const int l = __ldg(ls + ilm);
  if (l < 0 || l >= lsize) {
    for (int r = blockIdx.y; r < nr; r += gridDim.y) out[int64_t(r) * nlm + ilm] = make_double2(0.0, 0.0);
    return;
  }
  const double2 h0 = __ldg(h + ilm);
  const double2 h1 = npol > 1 ? __ldg(h + nlm + ilm) : make_double2(0.0, 0.0);
  for (int r = blockIdx.y; r < nr; r += gridDim.y) {
    const double f0 = __ldg(flX + (int64_t(l) * npol) * nr + r);
    double2 v;
    if (npol == 1) {
      v = make_double2(f0 * h0.x * weight, f0 * h0.y * weight);
    } else {
      const double f1 = __ldg(flX + (int64_t(l) * npol + 1) * nr + r);
      v = make_double2((f0 * h0.x + f1 * h1.x) * weight, (f0 * h0.y + f1 * h1.y) * weight);
    }
    out[int64_t(r) * nlm + ilm] = v;
  }
}

// out[X][lm] = Sum_r lm_map[r][lm] flXs[l][X][r] w[r]                       (tauNL_utils.pyx:220-237)
// spin1: 0.5 Sum_r (lm_map[0][r][lm] - lm_map[1][r][lm]) flXs[l][X][r] w[r]  (tauNL_utils.pyx:240-255)
__global__ void radial_sum_lm_kernel(const double2* __restrict__ lm_map, int spin1, const double* __restrict__ w,
                                     const double* __restrict__ flXs, int lsize, int npol, int nr,
                                     const int* __restrict__ ls, int64_t nlm, double2* __restrict__ out) {
  const int64_t ilm = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (ilm >= nlm) return;
  const int l = __ldg(ls + ilm);
  if (l < 0 || l >= lsize) {
    for (int X = 0; X < npol; ++X) out[int64_t(X) * nlm + ilm] = make_double2(0.0, 0.0);
    return;
  }
  for (int X = 0; X < npol; ++X) {
    double sx = 0.0, sy = 0.0;
    for (int r = 0; r < nr; ++r) {
      double2 v = __ldg(lm_map + int64_t(r) * nlm + ilm);
      if (spin1) {
        const double2 u = __ldg(lm_map + (int64_t(nr) + r) * nlm + ilm);
        v.x -= u.x;
        v.y -= u.y;
      }
      const double f = __ldg(flXs + (int64_t(l) * npol + X) * nr + r) * __ldg(w + r);
      sx += v.x * f;
      sy += v.y * f;
    }
    if (spin1) { sx *= 0.5; sy *= 0.5; }
    out[int64_t(X) * nlm + ilm] = make_double2(sx, sy);
  }
}

// ------------------------------------------------------------------ Fisher outer product
// fish[a][b] = Re Sum_j Sum_pq c_pq conj(Qa[p][a][j]) Qb[q][b][j] / (24 * 48)
// with c = [[1, 0, 0, -3], [0, 1, -3, 0], [0, -3, 9, 0], [-3, 0, 0, 9]]   (ideal_fisher.pyx:436-458)
constexpr int OP_T = 16;   // (a, b) tile
constexpr int OP_J = 16;   // j tile staged in shared memory
constexpr int OP_MAX_CHUNKS = 256;

__global__ void __launch_bounds__(OP_T* OP_T) outer_stage1(const double2* __restrict__ Qa, const double2* __restrict__ Qb,
                                                        int na, int nb, int64_t nin, int64_t per, int sym,
                                                        double* __restrict__ partial) {
  const int ta = blockIdx.y * OP_T, tb = blockIdx.z * OP_T;
  if (sym && ta > tb + OP_T - 1) return;  // tile entirely below the diagonal
  __shared__ double2 sA[4][OP_T][OP_J + 1];
  __shared__ double2 sB[4][OP_T][OP_J + 1];  // c applied: sB[p] = Sum_q c_pq Qb[q]
  const int tx = threadIdx.x % OP_T, ty = threadIdx.x / OP_T;  // (b, a) within the tile
  const int64_t j0 = int64_t(blockIdx.x) * per, j1 = min(nin, j0 + per);
  double acc = 0.0;
  for (int64_t jt = j0; jt < j1; jt += OP_J) {
    // load: thread (ty, tx) loads row ty, column jt + tx for all four components
    {
      const int row = ty, col = tx;
      const int64_t j = jt + col;
      const bool jok = j < j1;
#pragma unroll
      for (int p = 0; p < 4; ++p) {
        const int ra = ta + row;
        sA[p][row][col] = (jok && ra < na) ? __ldg(Qa + (int64_t(p) * na + ra) * nin + j) : make_double2(0.0, 0.0);
      }
      const int rb = tb + row;
      double2 q[4];
#pragma unroll
      for (int p = 0; p < 4; ++p)
        q[p] = (jok && rb < nb) ? __ldg(Qb + (int64_t(p) * nb + rb) * nin + j) : make_double2(0.0, 0.0);
      sB[0][row][col] = make_double2(q[0].x - 3 * q[3].x, q[0].y - 3 * q[3].y);
      sB[1][row][col] = make_double2(q[1].x - 3 * q[2].x, q[1].y - 3 * q[2].y);
      sB[2][row][col] = make_double2(9 * q[2].x - 3 * q[1].x, 9 * q[2].y - 3 * q[1].y);
      sB[3][row][col] = make_double2(9 * q[3].x - 3 * q[0].x, 9 * q[3].y - 3 * q[0].y);
    }
    __syncthreads();
#pragma unroll 4
    for (int jj = 0; jj < OP_J; ++jj) {
#pragma unroll
      for (int p = 0; p < 4; ++p) acc += re_conj_mul(sA[p][ty][jj], sB[p][tx][jj]);
    }
    __syncthreads();
  }
  const int a = ta + ty, b = tb + tx;
  if (a < na && b < nb) partial[(int64_t(blockIdx.x) * na + a) * nb + b] = acc;
}

__global__ void outer_stage2(const double* __restrict__ partial, int nchunks, int na, int nb, int sym,
                             double* __restrict__ fish) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= na * nb) return;
  const int a = idx / nb, b = idx % nb;
  if (sym && a > b) {
    double t = 0.0;  // mirror of (b, a), summed in the same order
    for (int c = 0; c < nchunks; ++c) t += partial[(int64_t(c) * na + b) * nb + a];
    fish[idx] = t / 24. / 48.;
    return;
  }
  double t = 0.0;
  for (int c = 0; c < nchunks; ++c) t += partial[(int64_t(c) * na + a) * nb + b];
  fish[idx] = t / 24. / 48.;
}

int outer_chunks(int na, int nb, int64_t nin) {
  const int tiles = ((na + OP_T - 1) / OP_T) * ((nb + OP_T - 1) / OP_T);
  int c = (sm_count() * 4 + tiles - 1) / tiles;
  const int64_t maxc = (nin + 1023) / 1024;
  if (c > maxc) c = int(maxc);
  if (c > OP_MAX_CHUNKS) c = OP_MAX_CHUNKS;
  return c < 1 ? 1 : c;
}

}  // namespace
}  // namespace ps

using namespace ps;

extern "C" int ps_pix_product(int op, const void* const* inputs, int n_inputs, void* out, int64_t n, int npol,
                              double fac, cudaStream_t stream) {
  const OpInfo info = op_info(op, npol);
  if (info.n_in < 0 || n_inputs != info.n_in || n < 0) return PS_ERR_INVALID;
  if ((op == PS_PIX_LENS_PHI || op == PS_PIX_LENS_PHI_SYM) ? (npol != 1 && npol != 3) : (npol != 1))
    return PS_ERR_INVALID;
  if (n == 0) return PS_OK;  // empty maps: nothing to read or write
  if (!inputs || !out) return PS_ERR_INVALID;
  PixIn a{};
  for (int k = 0; k < n_inputs; ++k) {
    if (!inputs[k]) return PS_ERR_INVALID;
    a.p[k] = inputs[k];
  }
  a.out = out;
  a.n = n;
  a.npol = npol;
  a.fac = fac;
  StatScope sc(PS_K_PIXEL, 0.0, info.bytes_per_elem * double(n), stream);
  const int grid = grid_for(n, sm_count());
  switch (op) {
    case PS_PIX_MULTIPLY: launch_op<PS_PIX_MULTIPLY>(a, grid, stream); break;
    case PS_PIX_MULTIPLY_ASYM: launch_op<PS_PIX_MULTIPLY_ASYM>(a, grid, stream); break;
    case PS_PIX_MULTIPLYC: launch_op<PS_PIX_MULTIPLYC>(a, grid, stream); break;
    case PS_PIX_MULTIPLYC_ASYM: launch_op<PS_PIX_MULTIPLYC_ASYM>(a, grid, stream); break;
    case PS_PIX_MULTIPLYCC: launch_op<PS_PIX_MULTIPLYCC>(a, grid, stream); break;
    case PS_PIX_MULTIPLYCC_ASYM: launch_op<PS_PIX_MULTIPLYCC_ASYM>(a, grid, stream); break;
    case PS_PIX_MULTIPLY2: launch_op<PS_PIX_MULTIPLY2>(a, grid, stream); break;
    case PS_PIX_MULTIPLY2R: launch_op<PS_PIX_MULTIPLY2R>(a, grid, stream); break;
    case PS_PIX_MULTIPLY2C: launch_op<PS_PIX_MULTIPLY2C>(a, grid, stream); break;
    case PS_PIX_MULTIPLYRC: launch_op<PS_PIX_MULTIPLYRC>(a, grid, stream); break;
    case PS_PIX_MULTIPLYRCSTAR: launch_op<PS_PIX_MULTIPLYRCSTAR>(a, grid, stream); break;
    case PS_PIX_MULTIPLYRC_SYM: launch_op<PS_PIX_MULTIPLYRC_SYM>(a, grid, stream); break;
    case PS_PIX_MULTIPLYRCSTAR_SYM: launch_op<PS_PIX_MULTIPLYRCSTAR_SYM>(a, grid, stream); break;
    case PS_PIX_MULTIPLYRR: launch_op<PS_PIX_MULTIPLYRR>(a, grid, stream); break;
    case PS_PIX_MULTIPLYRR_SYM: launch_op<PS_PIX_MULTIPLYRR_SYM>(a, grid, stream); break;
    case PS_PIX_R2C: launch_op<PS_PIX_R2C>(a, grid, stream); break;
    case PS_PIX_R2CSTAR: launch_op<PS_PIX_R2CSTAR>(a, grid, stream); break;
    case PS_PIX_LENS_PHI: launch_op<PS_PIX_LENS_PHI>(a, grid, stream); break;
    case PS_PIX_LENS_PHI_SYM: launch_op<PS_PIX_LENS_PHI_SYM>(a, grid, stream); break;
    case PS_PIX_PRODUCT_REAL1: launch_op<PS_PIX_PRODUCT_REAL1>(a, grid, stream); break;
    case PS_PIX_PRODUCT_REAL2: launch_op<PS_PIX_PRODUCT_REAL2>(a, grid, stream); break;
    default: return PS_ERR_INVALID;
  }
  PS_LAUNCH_CHECK();
  return PS_OK;
}

extern "C" int ps_pix_radial_sum_workspace_bytes(int nr, int64_t npix, size_t* bytes) {
  if (!bytes || nr <= 0 || npix <= 0) return PS_ERR_INVALID;
  *bytes = sizeof(double) * size_t(nr) * size_t(sum_chunks(nr, npix));
  return PS_OK;
}

extern "C" int ps_pix_radial_sum(int kind, const double* r_weights, const double* tau, const void* const* maps,
                                 int n_maps, int nr, int64_t npix, double* out, void* workspace,
                                 size_t workspace_bytes, cudaStream_t stream) {
  const SumInfo info = sum_info(kind);
  if (info.n_maps < 0 || n_maps != info.n_maps || !maps || !r_weights || !out || nr <= 0 || npix <= 0)
    return PS_ERR_INVALID;
  if (info.tpow > 0 && !tau) return PS_ERR_INVALID;
  SumIn a{};
  for (int k = 0; k < n_maps; ++k) {
    if (!maps[k]) return PS_ERR_INVALID;
    a.p[k] = maps[k];
  }
  a.npix = npix;
  a.nchunks = sum_chunks(nr, npix);
  if (!workspace || workspace_bytes < sizeof(double) * size_t(nr) * size_t(a.nchunks)) return PS_ERR_WORKSPACE;
  double* partial = static_cast<double*>(workspace);
  {
    StatScope sc(PS_K_PIXEL, 0.0, info.bytes_pix * double(nr) * double(npix), stream);
    switch (kind) {
      case PS_SUM_GNL_LOC: launch_sum<PS_SUM_GNL_LOC>(a, nr, partial, stream); break;
      case PS_SUM_GNL_LOC_DISC: launch_sum<PS_SUM_GNL_LOC_DISC>(a, nr, partial, stream); break;
      case PS_SUM_GNL_CON: launch_sum<PS_SUM_GNL_CON>(a, nr, partial, stream); break;
      case PS_SUM_GNL_CON_DISC: launch_sum<PS_SUM_GNL_CON_DISC>(a, nr, partial, stream); break;
      case PS_SUM_GNL_DOTDOT: launch_sum<PS_SUM_GNL_DOTDOT>(a, nr, partial, stream); break;
      case PS_SUM_GNL_DOTDOT_DISC: launch_sum<PS_SUM_GNL_DOTDOT_DISC>(a, nr, partial, stream); break;
      case PS_SUM_GNL_DOTDEL: launch_sum<PS_SUM_GNL_DOTDEL>(a, nr, partial, stream); break;
      case PS_SUM_GNL_DOTDEL_DISC: launch_sum<PS_SUM_GNL_DOTDEL_DISC>(a, nr, partial, stream); break;
      case PS_SUM_GNL_DELDEL: launch_sum<PS_SUM_GNL_DELDEL>(a, nr, partial, stream); break;
      case PS_SUM_GNL_DELDEL_DISC: launch_sum<PS_SUM_GNL_DELDEL_DISC>(a, nr, partial, stream); break;
      default: return PS_ERR_INVALID;
    }
    PS_LAUNCH_CHECK();
  }
  StatScope sc(PS_K_PIXEL, 0.0, 8.0 * nr * a.nchunks, stream);
  radial_sum_stage2<<<1, 256, 0, stream>>>(partial, r_weights, tau, info.tpow, nr, a.nchunks, out);
  PS_LAUNCH_CHECK();
  return PS_OK;
}

extern "C" int ps_apply_fl_weights(const double* flX, int lsize, int npol, int nr, const double* h_lm,
                                   const int* ls, int64_t nlm, double weight, double* out, cudaStream_t stream) {
  if (!flX || !h_lm || !ls || !out || lsize <= 0 || nr <= 0 || nlm < 0 || npol < 1 || npol > 3)
    return PS_ERR_INVALID;
  if (nlm == 0) return PS_OK;
  StatScope sc(PS_K_PIXEL, 0.0, 16.0 * nlm * (npol + nr) + 4.0 * nlm, stream);
  dim3 grid(unsigned((nlm + 255) / 256), unsigned(nr < 32 ? nr : 32));
  apply_fl_kernel<<<grid, 256, 0, stream>>>(flX, lsize, npol, nr, reinterpret_cast<const double2*>(h_lm), ls, nlm, weight,
                                             reinterpret_cast<double2*>(out));
  PS_LAUNCH_CHECK();
  return PS_OK;
}

extern "C" int ps_radial_sum_lm(const double* lm_map, int spin1, const double* r_weights, const double* flXs,
                                int lsize, int npol, int nr, const int* ls, int64_t nlm, double* out,
                                cudaStream_t stream) {
  if (!lm_map || !r_weights || !flXs || !ls || !out || lsize <= 0 || npol <= 0 || nr <= 0 || nlm < 0)
    return PS_ERR_INVALID;
  if (nlm == 0) return PS_OK;
  StatScope sc(PS_K_PIXEL, 0.0, 16.0 * nlm * (nr * (spin1 ? 2 : 1) + npol) + 4.0 * nlm, stream);
  radial_sum_lm_kernel<<<unsigned((nlm + 127) / 128), 128, 0, stream>>>(
      reinterpret_cast<const double2*>(lm_map), spin1 ? 1 : 0, r_weights, flXs, lsize, npol, nr, ls, nlm,
      reinterpret_cast<double2*>(out));
  PS_LAUNCH_CHECK();
  return PS_OK;
}

extern "C" int ps_outer_product_workspace_bytes(int na, int nb, int64_t nin, size_t* bytes) {
  if (!bytes || na <= 0 || nb <= 0 || nin <= 0) return PS_ERR_INVALID;
  *bytes = sizeof(double) * size_t(outer_chunks(na, nb, nin)) * size_t(na) * size_t(nb);
  return PS_OK;
}

extern "C" int ps_outer_product(const double* Qa, const double* Qb, int na, int nb, int64_t nin, int sym,
                                double* fish, void* workspace, size_t workspace_bytes, cudaStream_t stream) {
  if (!Qa || !Qb || !fish || na <= 0 || nb <= 0 || nin <= 0) return PS_ERR_INVALID;
  if (sym && na != nb) return PS_ERR_INVALID;
  const int nc = outer_chunks(na, nb, nin);
  if (!workspace || workspace_bytes < sizeof(double) * size_t(nc) * size_t(na) * size_t(nb)) return PS_ERR_WORKSPACE;
  const int64_t per = ((nin + nc - 1) / nc + OP_J - 1) / OP_J * OP_J;
  double* partial = static_cast<double*>(workspace);
  {
    StatScope sc(PS_K_PIXEL, 32.0 * na * double(nb) * nin, 64.0 * (na + nb) * double(nin), stream);
    dim3 grid(unsigned(nc), unsigned((na + OP_T - 1) / OP_T), unsigned((nb + OP_T - 1) / OP_T));
    outer_stage1<<<grid, OP_T * OP_T, 0, stream>>>(reinterpret_cast<const double2*>(Qa),
                                                    reinterpret_cast<const double2*>(Qb), na, nb, nin, per,
                                                    sym ? 1 : 0, partial);
    PS_LAUNCH_CHECK();
  }
  StatScope sc(PS_K_PIXEL, 0.0, 8.0 * nc * na * nb, stream);
  outer_stage2<<<unsigned((na * nb + 255) / 256), 256, 0, stream>>>(partial, nc, na, nb, sym ? 1 : 0, fish);
  PS_LAUNCH_CHECK();
  return PS_OK;
}
