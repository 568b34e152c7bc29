// Learned band preconditioner of the masked CG S^-1 filter: kernels for its
// training (moment accumulation from plain-CG (residual, error) pairs, the
// per-band loss and its gradient, a dense-layer forward/backward for the MLP,
// Adam) and for its application inside the CG.
//
// The preconditioner (no counterpart in the reference, whose CG offers the
// 'harmonic' and 'pseudo_inverse' preconditioners, polyspec/weighting.py:301-324):
//   M r = Sigma r + S^1/2 (L_b L_b^T + d_b I) S^1/2 r      on every band block b
// where Sigma is the harmonic preconditioner (per-l 3x3, weighting.py:76-78),
// S = diag(Sigma) per (field, lm), and a block b is (one m, LB consecutive l,
// the three fields T, E, B): D = 3 LB real coordinates, applied to the real and
// the imaginary parts of the alm alike.  L_b (D x K) and d_b = 0.5 tanh(q_b) are
// produced by a 3-layer MLP from features of the block (m, l, signal-to-noise,
// ...).  Sigma + d S is positive definite for |d| < 1 - rho, rho the largest
// correlation coefficient of the 3x3 Sigma (the T-E correlation, well below 0.5
// for CMB spectra), and L L^T adds a positive semi-definite term: M stays
// symmetric positive definite, so plain PCG remains valid.
//
// Training target: for plain-CG iterates x_k of a system with solution x*,
// e_k = x* - x_k solves A e_k = r_k; the loss is
//   J = Sum_s w_s || P u_s - t_s ||^2,  P = L L^T + d I,  u = S^1/2 r,  t = S^-1/2 (e - Sigma r)
// per block, i.e. the error of M r_k against e_k in the S^-1 norm.  With
// C = Sum w u u^T, G = Sym(Sum w u t^T), T = Sum w t^T t (accumulated once),
// A = L^T L, B = L^T C L, E = tr(L^T G L):
//   J_b = tr(B A) + 2 d tr(B) + d^2 tr(C) - 2 E - 2 d tr(G) + T
//   dJ_b/dL = 2 (C L A + L B + 2 d C L - 2 G L),  dJ_b/dd = 2 (tr(B) + d tr(C) - tr(G)).
// Layouts: C, G [nb][D][D] float32 (row-major, C and G symmetric); network
// output per block [D*K + 1] float32 (L row-major, then q); alm vectors
// complex128 [B][3][nalm] (m-major alm order).
#include <cuda_bf16.h>

#include "ps_common.cuh"
#include "ps_stats.cuh"

namespace ps {
namespace {

constexpr int LB = 16;        // l per band
constexpr int DB = 3 * LB;    // real coordinates per block (T, E, B)
constexpr int KR = 4;         // rank of the learned correction
constexpr int OUT = DB * KR + 1;  // network outputs per block: L, then q (d = 0.5 tanh q)
constexpr float D_MAX = 0.5f;

__device__ __forceinline__ float d_of_q(float q) { return D_MAX * tanhf(q); }

struct BlockDesc {
  const int64_t* idx0;  // alm index of (l0, m)
  const int* nl;        // number of valid l in the block (<= LB)
};

// ------------------------------------------------------------------ moments
// One CTA per block.  Samples: the real and imaginary parts of each of the B
// right-hand sides.  Sigma [3][3][nalm] float64 (symmetric per lm).
constexpr int MOM_THREADS = 256;
constexpr int MOM_PER_THREAD = (DB * DB + MOM_THREADS - 1) / MOM_THREADS;  // 9

__global__ void __launch_bounds__(MOM_THREADS) lbp_moments_kernel(
    BlockDesc bd, const double2* __restrict__ r, const double2* __restrict__ e, const double* __restrict__ w,
    const double* __restrict__ Sig, int B, int64_t nalm, float* __restrict__ C, float* __restrict__ G,
    float* __restrict__ T) {
  const int b = blockIdx.x;
  const int64_t i0 = bd.idx0[b];
  const int nl = bd.nl[b];
  __shared__ float su[2][DB], st[2][DB];
  float accC[MOM_PER_THREAD], accG[MOM_PER_THREAD];
#pragma unroll
  for (int q = 0; q < MOM_PER_THREAD; ++q) { accC[q] = 0.f; accG[q] = 0.f; }
  float accT = 0.f;
  for (int n = 0; n < B; ++n) {
    const float wn = float(w[n]);
    // thread j < DB builds coordinate j (field f = j / LB, l offset jl = j % LB) of u and t
    if (threadIdx.x < DB) {
      const int j = threadIdx.x, f = j / LB, jl = j % LB;
      float ur = 0.f, ui = 0.f, tr = 0.f, ti = 0.f;
      if (jl < nl) {
        const int64_t lm = i0 + jl;
        const double2 rf = r[(int64_t(n) * 3 + f) * nalm + lm];
        double sr = 0.0, si = 0.0;  // (Sigma r)_f
        for (int g = 0; g < 3; ++g) {
          const double s = Sig[(int64_t(f) * 3 + g) * nalm + lm];
          const double2 rg = r[(int64_t(n) * 3 + g) * nalm + lm];
          sr += s * rg.x;
          si += s * rg.y;
        }
        const double d = Sig[(int64_t(f) * 3 + f) * nalm + lm];
        const double sq = d > 0.0 ? sqrt(d) : 0.0, isq = d > 0.0 ? 1.0 / sqrt(d) : 0.0;
        const double2 ef = e[(int64_t(n) * 3 + f) * nalm + lm];
        ur = float(sq * rf.x);
        ui = float(sq * rf.y);
        tr = float(isq * (ef.x - sr));
        ti = float(isq * (ef.y - si));
      }
      su[0][j] = ur; su[1][j] = ui; st[0][j] = tr; st[1][j] = ti;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < MOM_PER_THREAD; ++q) {
      const int k = threadIdx.x + q * MOM_THREADS;
      if (k < DB * DB) {
        const int a = k / DB, c = k % DB;
        accC[q] += wn * (su[0][a] * su[0][c] + su[1][a] * su[1][c]);
        // symmetrised u t^T
        accG[q] += 0.5f * wn * (su[0][a] * st[0][c] + su[1][a] * st[1][c] + st[0][a] * su[0][c] + st[1][a] * su[1][c]);
      }
    }
    if (threadIdx.x < DB) {
      const int j = threadIdx.x;
      accT += wn * (st[0][j] * st[0][j] + st[1][j] * st[1][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < MOM_PER_THREAD; ++q) {
    const int k = threadIdx.x + q * MOM_THREADS;
    if (k < DB * DB) {
      C[int64_t(b) * DB * DB + k] += accC[q];
      G[int64_t(b) * DB * DB + k] += accG[q];
    }
  }
  // block total of t^T t (fixed order over the DB coordinates)
  __shared__ float sT[DB];
  if (threadIdx.x < DB) sT[threadIdx.x] = accT;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.f;
    for (int j = 0; j < DB; ++j) t += sT[j];
    T[b] += t;
  }
}

// ------------------------------------------------------------------ loss and dL
// One warp per block; lane holds rows lane and lane + 32 (< DB) of L, C L, G L.
constexpr int LG_WARPS = 4;

__global__ void __launch_bounds__(LG_WARPS * 32) lbp_loss_grad_kernel(const float* __restrict__ L,
                                                                    const float* __restrict__ C,
                                                                    const float* __restrict__ G,
                                                                    const float* __restrict__ T, int nb,
                                                                    float scale, float* __restrict__ dL,
                                                                    float* __restrict__ loss_blk) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int b = blockIdx.x * LG_WARPS + warp;
  __shared__ float sL[LG_WARPS][DB][KR];
  if (b >= nb) return;  // whole warp leaves together; no block-wide barrier below
  const float* Lb = L + int64_t(b) * OUT;
  for (int k = lane; k < DB * KR; k += 32) sL[warp][k / KR][k % KR] = Lb[k];
  const float q = Lb[DB * KR];
  const float dd = d_of_q(q);
  __syncwarp();
  const float* Cb = C + int64_t(b) * DB * DB;
  const float* Gb = G + int64_t(b) * DB * DB;
  float cl[2][KR], gl[2][KR], lr[2][KR];
  float trC = 0.f, trG = 0.f;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int row = lane + 32 * h;
    if (row < DB) { trC += Cb[row * DB + row]; trG += Gb[row * DB + row]; }
#pragma unroll
    for (int a = 0; a < KR; ++a) { cl[h][a] = 0.f; gl[h][a] = 0.f; lr[h][a] = 0.f; }
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    trC += __shfl_xor_sync(0xffffffffu, trC, off);
    trG += __shfl_xor_sync(0xffffffffu, trG, off);
  }
  for (int j = 0; j < DB; ++j) {
    // C and G are symmetric: row `row`, column j = C[j][row] (coalesced over lanes)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int row = lane + 32 * h;
      if (row < DB) {
        const float c = Cb[j * DB + row], g = Gb[j * DB + row];
#pragma unroll
        for (int a = 0; a < KR; ++a) {
          cl[h][a] += c * sL[warp][j][a];
          gl[h][a] += g * sL[warp][j][a];
        }
      }
    }
  }
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int row = lane + 32 * h;
#pragma unroll
    for (int a = 0; a < KR; ++a) lr[h][a] = row < DB ? sL[warp][row][a] : 0.f;
  }
  // A = L^T L, Bm = L^T C L, E = tr(L^T G L)
  float A[KR][KR], Bm[KR][KR], E = 0.f;
#pragma unroll
  for (int a = 0; a < KR; ++a)
#pragma unroll
    for (int c = 0; c < KR; ++c) {
      float va = 0.f, vb = 0.f;
#pragma unroll
      for (int h = 0; h < 2; ++h) { va += lr[h][a] * lr[h][c]; vb += lr[h][a] * cl[h][c]; }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        va += __shfl_xor_sync(0xffffffffu, va, off);
        vb += __shfl_xor_sync(0xffffffffu, vb, off);
      }
      A[a][c] = va;
      Bm[a][c] = vb;
    }
  {
    float ve = 0.f;
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
      for (int a = 0; a < KR; ++a) ve += lr[h][a] * gl[h][a];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) ve += __shfl_xor_sync(0xffffffffu, ve, off);
    E = ve;
  }
  float trBA = 0.f, trB = 0.f;
#pragma unroll
  for (int a = 0; a < KR; ++a) {
    trB += Bm[a][a];
#pragma unroll
    for (int c = 0; c < KR; ++c) trBA += Bm[a][c] * A[c][a];
  }
  if (lane == 0) {
    loss_blk[b] = trBA + 2.f * dd * trB + dd * dd * trC - 2.f * E - 2.f * dd * trG + T[b];
    const float dJdd = 2.f * (trB + dd * trC - trG);
    const float th = dd / D_MAX;
    dL[int64_t(b) * OUT + DB * KR] = dJdd * D_MAX * (1.f - th * th) * scale;
  }
  // dL = 2 (C L A + L B + 2 d C L - 2 G L) * scale
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int row = lane + 32 * h;
    if (row >= DB) continue;
#pragma unroll
    for (int c = 0; c < KR; ++c) {
      float v = -2.f * gl[h][c] + 2.f * dd * cl[h][c];
#pragma unroll
      for (int a = 0; a < KR; ++a) v += cl[h][a] * A[a][c] + lr[h][a] * Bm[a][c];
      dL[int64_t(b) * OUT + row * KR + c] = 2.f * v * scale;
    }
  }
}

// fixed-order sum of per-block values (one CTA)
__global__ void sum_fixed_kernel(const float* __restrict__ v, int n, double* __restrict__ out) {
  __shared__ double s[256];
  double acc = 0.0;
  const int per = (n + blockDim.x - 1) / blockDim.x;
  const int lo = threadIdx.x * per, hi = min(n, lo + per);
  for (int i = lo; i < hi; ++i) acc += double(v[i]);
  s[threadIdx.x] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int k = 0; k < int(blockDim.x); ++k) t += s[k];
    *out = t;
  }
}

// ------------------------------------------------------------------ dense layers
// Y[n][o] = act(Sum_i X[n][i] W[o][i] + bias[o]), W and bias bf16, X and Y float32,
// FP32 accumulation.  CTA: 32 rows (16 for the data gradient); X tile and W
// (bf16) staged in shared memory.
constexpr int DN_ROWS = 32;
constexpr int DB_ROWS = 16;
constexpr int DN_THREADS = 256;
constexpr int DN_MAXI = 64;
constexpr int DN_MAXO = 196;

__global__ void __launch_bounds__(DN_THREADS) dense_fwd_kernel(const float* __restrict__ X,
                                                             const __nv_bfloat16* __restrict__ W,
                                                             const __nv_bfloat16* __restrict__ bias, int n, int I,
                                                             int O, int relu, float* __restrict__ Y) {
  __shared__ float sX[DN_ROWS][DN_MAXI + 1];
  __shared__ __nv_bfloat16 sW[DN_MAXO][DN_MAXI + 2];
  const int r0 = blockIdx.x * DN_ROWS;
  for (int k = threadIdx.x; k < DN_ROWS * I; k += DN_THREADS) {
    const int rr = k / I, ii = k % I;
    sX[rr][ii] = (r0 + rr < n) ? X[int64_t(r0 + rr) * I + ii] : 0.f;
  }
  for (int k = threadIdx.x; k < O * I; k += DN_THREADS) sW[k / I][k % I] = W[k];
  __syncthreads();
  for (int k = threadIdx.x; k < DN_ROWS * O; k += DN_THREADS) {
    const int rr = k / O, o = k % O;
    if (r0 + rr >= n) continue;
    float acc = __bfloat162float(bias[o]);
    for (int i = 0; i < I; ++i) acc += sX[rr][i] * __bfloat162float(sW[o][i]);
    if (relu && acc < 0.f) acc = 0.f;
    Y[int64_t(r0 + rr) * O + o] = acc;
  }
}

// dZ = dY * act'(Y) (in place when relu); dX[n][i] = Sum_o dZ[n][o] W[o][i]
__global__ void __launch_bounds__(DN_THREADS) dense_bwd_data_kernel(float* __restrict__ dY,
                                                                  const float* __restrict__ Y,
                                                                  const __nv_bfloat16* __restrict__ W, int n, int I,
                                                                  int O, int relu, float* __restrict__ dX) {
  __shared__ float sD[DB_ROWS][DN_MAXO + 1];
  __shared__ __nv_bfloat16 sW[DN_MAXO][DN_MAXI + 2];
  const int r0 = blockIdx.x * DB_ROWS;
  for (int k = threadIdx.x; k < DB_ROWS * O; k += DN_THREADS) {
    const int rr = k / O, o = k % O;
    float d = 0.f;
    if (r0 + rr < n) {
      const int64_t g = int64_t(r0 + rr) * O + o;
      d = dY[g];
      if (relu && Y[g] <= 0.f) d = 0.f;
      dY[g] = d;
    }
    sD[rr][o] = d;
  }
  for (int k = threadIdx.x; k < O * I; k += DN_THREADS) sW[k / I][k % I] = W[k];
  __syncthreads();
  if (!dX) return;
  for (int k = threadIdx.x; k < DB_ROWS * I; k += DN_THREADS) {
    const int rr = k / I, i = k % I;
    if (r0 + rr >= n) continue;
    float acc = 0.f;
    for (int o = 0; o < O; ++o) acc += sD[rr][o] * __bfloat162float(sW[o][i]);
    dX[int64_t(r0 + rr) * I + i] = acc;
  }
}

// partial dW[c][o][i] = Sum_{n in chunk c} dZ[n][o] X[n][i], partial db[c][o]
constexpr int WG_CHUNK = 2048;
__global__ void dense_bwd_weight_kernel(const float* __restrict__ dZ, const float* __restrict__ X, int n, int I,
                                        int O, float* __restrict__ pW, float* __restrict__ pb) {
  const int c = blockIdx.x;
  const int lo = c * WG_CHUNK, hi = min(n, lo + WG_CHUNK);
  for (int k = threadIdx.x; k < O * I + O; k += blockDim.x) {
    float acc = 0.f;
    if (k < O * I) {
      const int o = k / I, i = k % I;
      for (int r = lo; r < hi; ++r) acc += dZ[int64_t(r) * O + o] * X[int64_t(r) * I + i];
      pW[int64_t(c) * O * I + k] = acc;
    } else {
      const int o = k - O * I;
      for (int r = lo; r < hi; ++r) acc += dZ[int64_t(r) * O + o];
      pb[int64_t(c) * O + o] = acc;
    }
  }
}

__global__ void sum_chunks_kernel(const float* __restrict__ p, int nchunks, int len, float* __restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= len) return;
  float acc = 0.f;
  for (int c = 0; c < nchunks; ++c) acc += p[int64_t(c) * len + k];
  out[k] = acc;
}

// Adam on FP32 master weights, bf16 copy for the forward pass
__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, __nv_bfloat16* __restrict__ pb, int n, float lr, float b1,
                            float b2, float eps, float c1, float c2) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const float gk = g[k];
  const float mk = b1 * m[k] + (1.f - b1) * gk;
  const float vk = b2 * v[k] + (1.f - b2) * gk * gk;
  m[k] = mk;
  v[k] = vk;
  const float pk = p[k] - lr * (mk / c1) / (sqrtf(vk / c2) + eps);
  p[k] = pk;
  pb[k] = __float2bfloat16(pk);
}

// ------------------------------------------------------------------ application
// z[n][f][lm] += S_f(lm)^1/2 ((L_b L_b^T + d_b I) u)_f,  u = S^1/2 r, real and imaginary parts
__global__ void __launch_bounds__(128) lbp_apply_kernel(BlockDesc bd, int nb, const float* __restrict__ L,
                                                        const double* __restrict__ Sig, const double2* __restrict__ r,
                                                        double2* __restrict__ z, int B, int64_t nalm) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int b = blockIdx.x * 4 + warp;
  if (b >= nb) return;
  const int64_t i0 = bd.idx0[b];
  const int nl = bd.nl[b];
  float lr[2][KR];
  double sq[2];
  int64_t off[2];
  bool ok[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int row = lane + 32 * h;
    const int f = row / LB, jl = row % LB;
    ok[h] = row < DB && jl < nl;
    off[h] = int64_t(f) * nalm + i0 + jl;
    sq[h] = 0.0;
    if (ok[h]) {
      const double d = Sig[(int64_t(f) * 3 + f) * nalm + i0 + jl];
      sq[h] = d > 0.0 ? sqrt(d) : 0.0;
    }
#pragma unroll
    for (int a = 0; a < KR; ++a) lr[h][a] = (row < DB) ? L[int64_t(b) * OUT + row * KR + a] : 0.f;
  }
  const float dd = d_of_q(L[int64_t(b) * OUT + DB * KR]);
  for (int n = 0; n < B; ++n) {
    double2 u[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      u[h] = make_double2(0.0, 0.0);
      if (ok[h]) {
        const double2 v = r[int64_t(n) * 3 * nalm + off[h]];
        u[h] = make_double2(sq[h] * v.x, sq[h] * v.y);
      }
    }
    float yr[KR], yi[KR];
#pragma unroll
    for (int a = 0; a < KR; ++a) {
      float sr = 0.f, si = 0.f;
#pragma unroll
      for (int h = 0; h < 2; ++h) { sr += lr[h][a] * float(u[h].x); si += lr[h][a] * float(u[h].y); }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        sr += __shfl_xor_sync(0xffffffffu, sr, o);
        si += __shfl_xor_sync(0xffffffffu, si, o);
      }
      yr[a] = sr;
      yi[a] = si;
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      if (!ok[h]) continue;
      float cr = dd * float(u[h].x), ci = dd * float(u[h].y);
#pragma unroll
      for (int a = 0; a < KR; ++a) { cr += lr[h][a] * yr[a]; ci += lr[h][a] * yi[a]; }
      double2* zp = z + int64_t(n) * 3 * nalm + off[h];
      double2 zv = *zp;
      zv.x += sq[h] * double(cr);
      zv.y += sq[h] * double(ci);
      *zp = zv;
    }
  }
}

bool dims_ok(int I, int O) { return I > 0 && O > 0 && I <= DN_MAXI && O <= DN_MAXO; }

}  // namespace
}  // namespace ps

using namespace ps;

extern "C" int ps_lbp_dims(int* lb, int* d, int* k, int* out) {
  if (!lb || !d || !k || !out) return PS_ERR_INVALID;
  *lb = LB;
  *d = DB;
  *k = KR;
  *out = OUT;
  return PS_OK;
}

extern "C" int ps_lbp_moments(const int64_t* blk_idx0, const int* blk_nl, int nb, const double* r, const double* e,
                              const double* w, const double* sigma, int batch, int64_t nalm, float* C, float* G,
                              float* T, cudaStream_t stream) {
  if (!blk_idx0 || !blk_nl || !r || !e || !w || !sigma || !C || !G || !T || nb <= 0 || batch <= 0 || nalm <= 0)
    return PS_ERR_INVALID;
  StatScope sc(PS_K_MLP, 4.0 * DB * DB * 2.0 * batch * nb, 8.0 * DB * DB * nb * 2.0 + 96.0 * batch * nalm, stream);
  lbp_moments_kernel<<<nb, MOM_THREADS, 0, stream>>>(BlockDesc{blk_idx0, blk_nl}, reinterpret_cast<const double2*>(r),
                                                     reinterpret_cast<const double2*>(e), w, sigma, batch, nalm, C, G,
                                                     T);
  PS_LAUNCH_CHECK();
  return PS_OK;
}

extern "C" int ps_lbp_loss_grad(const float* L, const float* C, const float* G, const float* T, int nb, float scale,
                                float* dL, float* loss_blk, double* loss, cudaStream_t stream) {
  if (!L || !C || !G || !T || !dL || !loss_blk || !loss || nb <= 0) return PS_ERR_INVALID;
  StatScope sc(PS_K_MLP, 4.0 * DB * DB * KR * nb, 8.0 * DB * DB * nb, stream);
  lbp_loss_grad_kernel<<<(nb + LG_WARPS - 1) / LG_WARPS, LG_WARPS * 32, 0, stream>>>(L, C, G, T, nb, scale, dL,
                                                                                       loss_blk);
  PS_LAUNCH_CHECK();
  sum_fixed_kernel<<<1, 256, 0, stream>>>(loss_blk, nb, loss);
  PS_LAUNCH_CHECK();
  return PS_OK;
}

extern "C" int ps_mlp_dense_forward(const float* X, const void* W_bf16, const void* b_bf16, int n, int in_dim,
                                    int out_dim, int relu, float* Y, cudaStream_t stream) {
  if (!X || !W_bf16 || !b_bf16 || !Y || n <= 0 || !dims_ok(in_dim, out_dim)) return PS_ERR_INVALID;
  StatScope sc(PS_K_MLP, 2.0 * n * in_dim * out_dim, 4.0 * n * (in_dim + out_dim), stream);
  dense_fwd_kernel<<<(n + DN_ROWS - 1) / DN_ROWS, DN_THREADS, 0, stream>>>(
      X, static_cast<const __nv_bfloat16*>(W_bf16), static_cast<const __nv_bfloat16*>(b_bf16), n, in_dim, out_dim,
      relu ? 1 : 0, Y);
  PS_LAUNCH_CHECK();
  return PS_OK;
}

extern "C" int ps_mlp_dense_backward_workspace_bytes(int n, int in_dim, int out_dim, size_t* bytes) {
  if (!bytes || n <= 0 || !dims_ok(in_dim, out_dim)) return PS_ERR_INVALID;
  const size_t nc = size_t((n + WG_CHUNK - 1) / WG_CHUNK);
  *bytes = sizeof(float) * nc * size_t(out_dim) * size_t(in_dim + 1);
  return PS_OK;
}

extern "C" int ps_mlp_dense_backward(float* dY, const float* Y, const float* X, const void* W_bf16, int n,
                                     int in_dim, int out_dim, int relu, float* dX, float* dW, float* db,
                                     void* workspace, size_t workspace_bytes, cudaStream_t stream) {
  if (!dY || !Y || !X || !W_bf16 || !dW || !db || n <= 0 || !dims_ok(in_dim, out_dim)) return PS_ERR_INVALID;
  const int nc = (n + WG_CHUNK - 1) / WG_CHUNK;
  const size_t need = sizeof(float) * size_t(nc) * size_t(out_dim) * size_t(in_dim + 1);
  if (!workspace || workspace_bytes < need) return PS_ERR_WORKSPACE;
  StatScope sc(PS_K_MLP, 4.0 * n * in_dim * out_dim, 4.0 * n * (2 * in_dim + 2 * out_dim), stream);
  dense_bwd_data_kernel<<<(n + DB_ROWS - 1) / DB_ROWS, DN_THREADS, 0, stream>>>(
      dY, Y, static_cast<const __nv_bfloat16*>(W_bf16), n, in_dim, out_dim, relu ? 1 : 0, dX);
  PS_LAUNCH_CHECK();
  float* pW = static_cast<float*>(workspace);
  float* pb = pW + size_t(nc) * out_dim * in_dim;
  dense_bwd_weight_kernel<<<nc, 256, 0, stream>>>(dY, X, n, in_dim, out_dim, pW, pb);
  PS_LAUNCH_CHECK();
  sum_chunks_kernel<<<(out_dim * in_dim + 255) / 256, 256, 0, stream>>>(pW, nc, out_dim * in_dim, dW);
  PS_LAUNCH_CHECK();
  sum_chunks_kernel<<<(out_dim + 255) / 256, 256, 0, stream>>>(pb, nc, out_dim, db);
  PS_LAUNCH_CHECK();
  return PS_OK;
}

extern "C" int ps_mlp_adam(float* param, const float* grad, float* m, float* v, void* param_bf16, int n, float lr,
                           float beta1, float beta2, float eps, int step, cudaStream_t stream) {
  if (!param || !grad || !m || !v || !param_bf16 || n <= 0 || step <= 0) return PS_ERR_INVALID;
  const float c1 = 1.f - powf(beta1, float(step)), c2 = 1.f - powf(beta2, float(step));
  StatScope sc(PS_K_MLP, 10.0 * n, 22.0 * n, stream);
  adam_kernel<<<(n + 255) / 256, 256, 0, stream>>>(param, grad, m, v, static_cast<__nv_bfloat16*>(param_bf16), n, lr,
                                                   beta1, beta2, eps, c1, c2);
  PS_LAUNCH_CHECK();
  return PS_OK;
}

extern "C" int ps_lbp_apply(const int64_t* blk_idx0, const int* blk_nl, int nb, const float* L, const double* sigma,
                            const double* r, double* z, int batch, int64_t nalm, cudaStream_t stream) {
  if (!blk_idx0 || !blk_nl || !L || !sigma || !r || !z || nb <= 0 || batch <= 0 || nalm <= 0) return PS_ERR_INVALID;
  StatScope sc(PS_K_MLP, 8.0 * OUT * batch * double(nb), 4.0 * OUT * nb + 96.0 * batch * nalm, stream);
  lbp_apply_kernel<<<(nb + 3) / 4, 128, 0, stream>>>(BlockDesc{blk_idx0, blk_nl}, nb, L, sigma,
                                                     reinterpret_cast<const double2*>(r), reinterpret_cast<double2*>(z),
                                                     batch, nalm);
  PS_LAUNCH_CHECK();
  return PS_OK;
}
