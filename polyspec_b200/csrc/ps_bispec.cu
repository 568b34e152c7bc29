// Binned-bispectrum kernels (BSpecBin, polyspec/bspec_bin.py), FP64.
//
//  * ps_bispec_triplet_sums: out[o] = Sum_pix Sum_{t in terms(o)} M[a_t] M[b_t] M[c_t]
//    over planar complex maps M [nmap][2][npix] (real plane, imaginary plane):
//    the per-triplet pixel sums of Bl_numerator's cubic and linear terms
//    (bspec_bin.py:339-364, 383-415) and Bl_numerator_ideal (:733-755), one
//    launch for every triplet instead of one pool task per triplet.  Each CTA
//    walks pixel tiles; a tile of every map is staged in shared memory (one read
//    of the maps per pass of 64 outputs); warp w keeps G = 8 outputs in registers,
//    lanes own pixels, so shared-memory reads are conflict-free.  Per-CTA partials
//    are added in a fixed order by a second kernel.
//  * ps_bispec_pair_products: out[k] = Sum_t s_t op_t(A[a_t]) B[b_t] (op = identity
//    or complex conjugate, s_t a signed small integer), written as planar [2][npix]
//    real maps -- the inputs of
//    the spin-2 and spin-1 adjoint transforms of the H-map products of
//    compute_fisher_contribution (bspec_bin.py:496-518).
//  * ps_bispec_assemble_q: the Q3 rows of compute_fisher_contribution
//    (bspec_bin.py:520-547): for every row, the sum of its (pair, field, l-bin)
//    contributions of conj(G1) - conj(G2) or conj(C1) + conj(C2), where (G2, C2),
//    (G1, C1) are the spin-2 and spin-1 adjoint outputs of the pair, times a
//    per-(field, lm) scale (the m weights or the beam); one write of each row.
#include "ps_common.cuh"
#include "ps_stats.cuh"

namespace ps {
namespace {

constexpr int TS_THREADS = 256;
constexpr int TS_WARPS = TS_THREADS / 32;
constexpr int TS_G = 8;                      // outputs per warp per pass
constexpr int TS_PASS = TS_WARPS * TS_G;     // outputs per pass
constexpr size_t TS_SMEM_SOFT = 110 * 1024;  // preferred staging size (2 CTAs per SM)
constexpr size_t TS_SMEM_MAX = 220 * 1024;

int ts_tile(int nmap) {
  for (int tp = 128; tp >= 32; tp >>= 1)
    if (size_t(nmap) * 2 * tp * sizeof(double) <= TS_SMEM_SOFT) return tp;
  if (size_t(nmap) * 2 * 32 * sizeof(double) <= TS_SMEM_MAX) return 32;
  return 0;
}

int n_sms_bs() {
  static int sms = 0;
  if (sms == 0) {
    int dev = 0, c = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, dev);
    sms = c > 0 ? c : 148;
  }
  return sms;
}

void ts_grid(int nmap, int64_t npix, int nout, int& tp, int& gx, int& npass) {
  tp = ts_tile(nmap);
  npass = (nout + TS_PASS - 1) / TS_PASS;
  if (tp == 0) { gx = 0; return; }
  const size_t smem = size_t(nmap) * 2 * tp * sizeof(double);
  int per_sm = int((228 * 1024) / (smem + 1024));
  if (per_sm > 2048 / TS_THREADS) per_sm = 2048 / TS_THREADS;
  if (per_sm < 1) per_sm = 1;
  const int64_t ntile = (npix + tp - 1) / tp;
  int64_t want = (int64_t(n_sms_bs()) * per_sm + npass - 1) / npass;
  if (want > ntile) want = ntile;
  if (want > 4096) want = 4096;
  gx = int(want < 1 ? 1 : want);
}

template <int TP>
__global__ void __launch_bounds__(TS_THREADS) triplet_stage1(const double* __restrict__ maps, int nmap, int64_t npix,
                                                             const int* __restrict__ term_ptr,
                                                             const int* __restrict__ terms, int nout,
                                                             double2* __restrict__ partial) {
  extern __shared__ __align__(16) double sm[];  // [nmap][2][TP]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int obase = blockIdx.y * TS_PASS + warp * TS_G;
  double2 acc[TS_G];
#pragma unroll
  for (int g = 0; g < TS_G; ++g) acc[g] = make_double2(0.0, 0.0);
  const int64_t ntile = (npix + TP - 1) / TP;
  const int nvec = nmap * TP;  // double2 words staged per tile (2 planes x TP / 2)
  for (int64_t tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
    const int64_t p0 = tile * TP;
    const int64_t n = min(int64_t(TP), npix - p0);  // even: npix and TP are even
    __syncthreads();
    for (int v = threadIdx.x; v < nvec; v += TS_THREADS) {
      const int plane = v / (TP / 2), p = 2 * (v - plane * (TP / 2));
      double2 w = make_double2(0.0, 0.0);
      if (p < n) w = __ldg(reinterpret_cast<const double2*>(maps + int64_t(plane) * npix + p0 + p));
      reinterpret_cast<double2*>(sm + plane * TP)[p >> 1] = w;
    }
    __syncthreads();
#pragma unroll
    for (int g = 0; g < TS_G; ++g) {
      const int o = obase + g;
      if (o >= nout) continue;  // uniform over the warp
      const int t0 = __ldg(term_ptr + o), t1 = __ldg(term_ptr + o + 1);
      for (int t = t0; t < t1; ++t) {
        const int a = __ldg(terms + 3 * t), b = __ldg(terms + 3 * t + 1), c = __ldg(terms + 3 * t + 2);
        if (unsigned(a) >= unsigned(nmap) || unsigned(b) >= unsigned(nmap) || unsigned(c) >= unsigned(nmap))
          continue;  // an index outside the map set contributes nothing
        const double* ma = sm + 2 * a * TP;
        const double* mb = sm + 2 * b * TP;
        const double* mc = sm + 2 * c * TP;
#pragma unroll
        for (int k = 0; k < TP / 32; ++k) {
          const int p = lane + 32 * k;
          const double2 x = make_double2(ma[p], ma[TP + p]);
          const double2 y = make_double2(mb[p], mb[TP + p]);
          const double2 z = make_double2(mc[p], mc[TP + p]);
          const double2 xy = cmul(x, y);
          acc[g].x = fma(xy.x, z.x, fma(-xy.y, z.y, acc[g].x));
          acc[g].y = fma(xy.x, z.y, fma(xy.y, z.x, acc[g].y));
        }
      }
    }
  }
#pragma unroll
  for (int g = 0; g < TS_G; ++g) {
    double x = acc[g].x, y = acc[g].y;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      x += __shfl_xor_sync(0xffffffffu, x, off);
      y += __shfl_xor_sync(0xffffffffu, y, off);
    }
    const int o = obase + g;
    if (lane == 0 && o < nout) partial[int64_t(blockIdx.x) * nout + o] = make_double2(x, y);
  }
}

__global__ void triplet_stage2(const double2* __restrict__ partial, int ncta, int nout, double2* __restrict__ out) {
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= nout) return;
  double x = 0.0, y = 0.0;
  for (int c = 0; c < ncta; ++c) {
    const double2 v = partial[int64_t(c) * nout + o];
    x += v.x;
    y += v.y;
  }
  out[o] = make_double2(x, y);
}

// out[k] planar [2][npix]; two pixels per thread (double2 words of each plane)
__global__ void pair_products_kernel(const double* __restrict__ A, int nA, const double* __restrict__ B, int nB,
                                     int64_t npix,
                                     const int* __restrict__ ptr, const int* __restrict__ prods,
                                     double* __restrict__ out) {
  const int k = blockIdx.y;
  const int t0 = __ldg(ptr + k), t1 = __ldg(ptr + k + 1);
  const int64_t half = npix >> 1;
  for (int64_t q = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; q < half; q += int64_t(gridDim.x) * blockDim.x) {
    double2 re = make_double2(0.0, 0.0), im = make_double2(0.0, 0.0);
    for (int t = t0; t < t1; ++t) {
      const int a = __ldg(prods + 3 * t), b = __ldg(prods + 3 * t + 1), f = __ldg(prods + 3 * t + 2);
      if (unsigned(a) >= unsigned(nA) || unsigned(b) >= unsigned(nB)) continue;
      const double2 ar = __ldg(reinterpret_cast<const double2*>(A + (2 * int64_t(a)) * npix) + q);
      double2 ai = __ldg(reinterpret_cast<const double2*>(A + (2 * int64_t(a) + 1) * npix) + q);
      const double2 br = __ldg(reinterpret_cast<const double2*>(B + (2 * int64_t(b)) * npix) + q);
      const double2 bi = __ldg(reinterpret_cast<const double2*>(B + (2 * int64_t(b) + 1) * npix) + q);
      if (f & 1) { ai.x = -ai.x; ai.y = -ai.y; }
      const int mult = (f >> 2) & 63;  // term multiplicity (0 means 1)
      const double s = ((f & 2) ? -1.0 : 1.0) * double(mult ? mult : 1);
      re.x = fma(s, ar.x * br.x - ai.x * bi.x, re.x);
      re.y = fma(s, ar.y * br.y - ai.y * bi.y, re.y);
      im.x = fma(s, ar.x * bi.x + ai.x * br.x, im.x);
      im.y = fma(s, ar.y * bi.y + ai.y * br.y, im.y);
    }
    reinterpret_cast<double2*>(out + (2 * int64_t(k)) * npix)[q] = re;
    reinterpret_cast<double2*>(out + (2 * int64_t(k) + 1) * npix)[q] = im;
  }
}

// contrib[c] = {pair, field, bin, which}: which 0 -> conj(G1) - conj(G2), 1 -> conj(C1) + conj(C2)
__global__ void assemble_q_kernel(const double2* __restrict__ A2, const double2* __restrict__ A1, int npair,
                                  int64_t nlm, const int* __restrict__ l_of_lm, const int* __restrict__ edges,
                                  int nbins,
                                  const int* __restrict__ row_ptr, const int* __restrict__ contrib,
                                  const double* __restrict__ coef, int nfield, const double* __restrict__ scale,
                                  double2* __restrict__ out) {
  const int r = blockIdx.y;
  const int c0 = __ldg(row_ptr + r), c1 = __ldg(row_ptr + r + 1);
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < nlm; i += int64_t(gridDim.x) * blockDim.x) {
    const int l = __ldg(l_of_lm + i);
    for (int u = 0; u < nfield; ++u) {
      double x = 0.0, y = 0.0;
      for (int c = c0; c < c1; ++c) {
        if (__ldg(contrib + 4 * c + 1) != u) continue;
        const int b = __ldg(contrib + 4 * c + 2);
        const int kk = __ldg(contrib + 4 * c);
        const int which = __ldg(contrib + 4 * c + 3);
        if (unsigned(b) >= unsigned(nbins) || unsigned(kk) >= unsigned(npair) || unsigned(which) > 1u) continue;
        if (l < __ldg(edges + b) || l >= __ldg(edges + b + 1)) continue;
        const int64_t k = kk;
        const double2 v2 = A2 ? __ldg(A2 + (2 * k + which) * nlm + i) : make_double2(0.0, 0.0);
        const double2 v1 = __ldg(A1 + (2 * k + which) * nlm + i);
        const double w = __ldg(coef + c);
        if (which == 0) {  // conj(G1) - conj(G2)
          x = fma(w, v1.x - v2.x, x);
          y = fma(w, v2.y - v1.y, y);
        } else {  // conj(C1) + conj(C2)
          x = fma(w, v1.x + v2.x, x);
          y = fma(w, -(v1.y + v2.y), y);
        }
      }
      const double s = scale ? __ldg(scale + int64_t(u) * nlm + i) : 1.0;
      out[(int64_t(r) * nfield + u) * nlm + i] = make_double2(x * s, y * s);
    }
  }
}

}  // namespace
}  // namespace ps

using namespace ps;

extern "C" int ps_bispec_triplet_sums_workspace_bytes(int nmap, int64_t npix, int nout, size_t* bytes) {
  if (!bytes || nmap <= 0 || npix <= 0 || nout <= 0) return PS_ERR_INVALID;
  int tp, gx, npass;
  ts_grid(nmap, npix, nout, tp, gx, npass);
  if (tp == 0) return PS_ERR_UNSUPPORTED;
  *bytes = sizeof(double2) * size_t(gx) * size_t(nout);
  return PS_OK;
}

extern "C" int ps_bispec_triplet_sums(const double* maps, int nmap, int64_t npix, const int* term_ptr,
                                      const int* terms, int nout, double* out, void* workspace,
                                      size_t workspace_bytes, cudaStream_t stream) {
  if (nout == 0) return PS_OK;
  if (!maps || !term_ptr || !terms || !out || nmap <= 0 || npix <= 0 || nout < 0 || (npix & 1)) return PS_ERR_INVALID;
  if (reinterpret_cast<uintptr_t>(maps) & 15) return PS_ERR_INVALID;
  int tp, gx, npass;
  ts_grid(nmap, npix, nout, tp, gx, npass);
  if (tp == 0) return PS_ERR_UNSUPPORTED;
  if (!workspace || workspace_bytes < sizeof(double2) * size_t(gx) * size_t(nout)) return PS_ERR_WORKSPACE;
  const size_t smem = size_t(nmap) * 2 * tp * sizeof(double);
  double2* partial = static_cast<double2*>(workspace);
  // flops: ~10 per term per pixel (two complex products and the accumulation)
  StatScope sc(PS_K_PIXEL, 0.0, double(npass) * nmap * 16.0 * npix, stream);
  const dim3 grid(gx, npass);
  cudaError_t e;
  switch (tp) {
    case 128:
      e = cudaFuncSetAttribute(triplet_stage1<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
      if (e != cudaSuccess) return PS_ERR_CUDA;
      triplet_stage1<128><<<grid, TS_THREADS, smem, stream>>>(maps, nmap, npix, term_ptr, terms, nout, partial);
      break;
    case 64:
      e = cudaFuncSetAttribute(triplet_stage1<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
      if (e != cudaSuccess) return PS_ERR_CUDA;
      triplet_stage1<64><<<grid, TS_THREADS, smem, stream>>>(maps, nmap, npix, term_ptr, terms, nout, partial);
      break;
    default:
      e = cudaFuncSetAttribute(triplet_stage1<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
      if (e != cudaSuccess) return PS_ERR_CUDA;
      triplet_stage1<32><<<grid, TS_THREADS, smem, stream>>>(maps, nmap, npix, term_ptr, terms, nout, partial);
      break;
  }
  PS_LAUNCH_CHECK();
  triplet_stage2<<<(nout + 127) / 128, 128, 0, stream>>>(partial, gx, nout, reinterpret_cast<double2*>(out));
  PS_LAUNCH_CHECK();
  return PS_OK;
}

extern "C" int ps_bispec_pair_products(const double* A, int nA, const double* B, int nB, int64_t npix,
                                       const int* ptr, const int* prods, int nout, double* out,
                                       cudaStream_t stream) {
  if (nout == 0) return PS_OK;
  if (!A || !B || !ptr || !prods || !out || nA <= 0 || nB <= 0 || npix <= 0 || nout < 0 || (npix & 1))
    return PS_ERR_INVALID;
  if ((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B) | reinterpret_cast<uintptr_t>(out)) & 15)
    return PS_ERR_INVALID;
  if (nout > 65535) return PS_ERR_INVALID;
  StatScope sc(PS_K_PIXEL, 0.0, double(nout) * 16.0 * npix * 3.0, stream);
  const int64_t half = npix >> 1;
  int64_t gx = (half + 255) / 256;
  const int64_t cap = (int64_t(n_sms_bs()) * 8 + nout - 1) / nout;
  if (gx > cap) gx = cap < 1 ? 1 : cap;
  pair_products_kernel<<<dim3(unsigned(gx), nout), 256, 0, stream>>>(A, nA, B, nB, npix, ptr, prods, out);
  PS_LAUNCH_CHECK();
  return PS_OK;
}

extern "C" int ps_bispec_assemble_q(const double* A2, const double* A1, int npair, int64_t nlm,
                                    const int* l_of_lm, const int* edges, int nbins, const int* row_ptr,
                                    const int* contrib, const double* coef, int nrow, int nfield,
                                    const double* scale, double* out, cudaStream_t stream) {
  if (nrow == 0) return PS_OK;
  if (!A1 || !l_of_lm || !edges || !row_ptr || !contrib || !coef || !out || npair <= 0 || nlm <= 0 ||
      nbins <= 0 || nrow < 0 || nfield < 1 || nfield > 3 || nrow > 65535)
    return PS_ERR_INVALID;
  StatScope sc(PS_K_VECTOR, 0.0, double(nrow) * nfield * 16.0 * nlm, stream);
  int64_t gx = (nlm + 255) / 256;
  const int64_t cap = (int64_t(n_sms_bs()) * 8 + nrow - 1) / nrow;
  if (gx > cap) gx = cap < 1 ? 1 : cap;
  assemble_q_kernel<<<dim3(unsigned(gx), nrow), 256, 0, stream>>>(
      reinterpret_cast<const double2*>(A2), reinterpret_cast<const double2*>(A1), npair, nlm, l_of_lm, edges, nbins,
      row_ptr, contrib, coef, nfield, scale, reinterpret_cast<double2*>(out));
  PS_LAUNCH_CHECK();
  return PS_OK;
}
