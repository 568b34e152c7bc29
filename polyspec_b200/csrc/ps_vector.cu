// Harmonic-space vector kernels of the CG S^-1 filter (FP64, HBM-bound).
//
//  * ps_lm_matvec3:  y[n][a][i] = post[a][i] * Sum_b S[a][b][i] * pre[b][i] * x[n][b][i]
//    for per-(l, m) real 3x3 matrices S (the harmonic preconditioner Sigma of
//    polyspec/weighting.py:76-78, the inverse signal covariance C^-1 of :60-68)
//    and optional per-(field, lm) real scales (the beam), on complex128
//    vectors [B][3][nalm]: one read of x and S, one write of y.
//  * ps_lm_dot:  out[n] = Sum_{a,i} w[i] Re(x[n][a][i] conj(y[n][a][i])) -- the
//    CG's m-weighted inner product (weighting.py:255) -- by a grid-stride pass
//    into per-CTA partials and a fixed-order final sum per batch member.
#include "ps_common.cuh"
#include "ps_stats.cuh"

namespace ps {
namespace {

__global__ void lm_matvec3_kernel(const double* __restrict__ S, const double* __restrict__ pre,
                                  const double* __restrict__ post, const double2* __restrict__ x,
                                  double2* __restrict__ y, int B, int64_t nalm) {
  const int64_t total = int64_t(B) * nalm;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total; t += int64_t(gridDim.x) * blockDim.x) {
    const int64_t n = t / nalm, i = t - n * nalm;
    double2 v[3];
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      v[b] = x[(n * 3 + b) * nalm + i];
      if (pre) {
        const double s = pre[int64_t(b) * nalm + i];
        v[b].x *= s;
        v[b].y *= s;
      }
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      double re = 0.0, im = 0.0;
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        const double s = __ldg(S + (int64_t(a) * 3 + b) * nalm + i);
        re = fma(s, v[b].x, re);
        im = fma(s, v[b].y, im);
      }
      if (post) {
        const double s = post[int64_t(a) * nalm + i];
        re *= s;
        im *= s;
      }
      y[(n * 3 + a) * nalm + i] = make_double2(re, im);
    }
  }
}

constexpr int DOT_THREADS = 256;

// partial[n][c]: CTA c's share of batch member n
__global__ void lm_dot_stage1(const double2* __restrict__ x, const double2* __restrict__ y,
                              const double* __restrict__ w, int64_t nalm, int nchunks, double* __restrict__ partial) {
  const int n = blockIdx.y, c = blockIdx.x;
  const int64_t len = 3 * nalm;
  const int64_t per = (len + nchunks - 1) / nchunks;
  const int64_t lo = int64_t(c) * per, hi = min(len, lo + per);
  const double2* xn = x + int64_t(n) * len;
  const double2* yn = y + int64_t(n) * len;
  double acc = 0.0;
  for (int64_t k = lo + threadIdx.x; k < hi; k += DOT_THREADS) {
    const int64_t i = k % nalm;
    const double2 a = xn[k], b = yn[k];
    acc += __ldg(w + i) * (a.x * b.x + a.y * b.y);
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
  __shared__ double sw[DOT_THREADS / 32];
  if ((threadIdx.x & 31) == 0) sw[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int k = 0; k < DOT_THREADS / 32; ++k) t += sw[k];
    partial[int64_t(n) * nchunks + c] = t;
  }
}

__global__ void lm_dot_stage2(const double* __restrict__ partial, int B, int nchunks, double* __restrict__ out) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= B) return;
  double t = 0.0;
  for (int c = 0; c < nchunks; ++c) t += partial[int64_t(n) * nchunks + c];
  out[n] = t;
}

// y[n][a][i] += Sum_b S[a][b][i] x[n][b][i]  (y may not alias x)
__global__ void lm_matvec3_add_kernel(const double* __restrict__ S, const double2* __restrict__ x,
                                      double2* __restrict__ y, int B, int64_t nalm) {
  const int64_t total = int64_t(B) * nalm;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total; t += int64_t(gridDim.x) * blockDim.x) {
    const int64_t n = t / nalm, i = t - n * nalm;
    double2 v[3];
#pragma unroll
    for (int b = 0; b < 3; ++b) v[b] = x[(n * 3 + b) * nalm + i];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      double2 acc = y[(n * 3 + a) * nalm + i];
#pragma unroll
      for (int b = 0; b < 3; ++b) acc = cfma(__ldg(S + (int64_t(a) * 3 + b) * nalm + i), v[b], acc);
      y[(n * 3 + a) * nalm + i] = acc;
    }
  }
}

// partial[n][c] of Sum w[i] Re(x conj(S x)) (the quadratic form, S x never stored)
__global__ void lm_quad_stage1(const double* __restrict__ S, const double2* __restrict__ x,
                               const double* __restrict__ w, int64_t nalm, int nchunks, double* __restrict__ partial) {
  const int n = blockIdx.y, c = blockIdx.x;
  const int64_t per = (nalm + nchunks - 1) / nchunks;
  const int64_t lo = int64_t(c) * per, hi = min(nalm, lo + per);
  const double2* xn = x + int64_t(n) * 3 * nalm;
  double acc = 0.0;
  for (int64_t i = lo + threadIdx.x; i < hi; i += DOT_THREADS) {
    double2 v[3];
#pragma unroll
    for (int b = 0; b < 3; ++b) v[b] = xn[int64_t(b) * nalm + i];
    double q = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      double2 sx = make_double2(0.0, 0.0);
#pragma unroll
      for (int b = 0; b < 3; ++b) sx = cfma(__ldg(S + (int64_t(a) * 3 + b) * nalm + i), v[b], sx);
      q += v[a].x * sx.x + v[a].y * sx.y;
    }
    acc = fma(__ldg(w + i), q, acc);
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
  __shared__ double sw[DOT_THREADS / 32];
  if ((threadIdx.x & 31) == 0) sw[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int k = 0; k < DOT_THREADS / 32; ++k) t += sw[k];
    partial[int64_t(n) * nchunks + c] = t;
  }
}

// x[slot[n]] += alpha[n] p[n];  r[n] -= alpha[n] q[n]   (rows of `per` complex values)
__global__ void cg_xr_kernel(double2* __restrict__ x, const int64_t* __restrict__ slot,
                             const double* __restrict__ alpha, const double2* __restrict__ p, double2* __restrict__ r,
                             const double2* __restrict__ q, int B, int64_t per) {
  const int64_t total = int64_t(B) * per;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total; t += int64_t(gridDim.x) * blockDim.x) {
    const int64_t n = t / per, k = t - n * per;
    const double a = alpha[n];
    const int64_t xs = (slot ? slot[n] : n) * per + k;
    x[xs] = cfma(a, p[t], x[xs]);
    r[t] = cfma(-a, q[t], r[t]);
  }
}

// p[n] = z[n] + beta[n] p[n]
__global__ void cg_dir_kernel(double2* __restrict__ p, const double2* __restrict__ z, const double* __restrict__ beta,
                              int B, int64_t per) {
  const int64_t total = int64_t(B) * per;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total; t += int64_t(gridDim.x) * blockDim.x)
    p[t] = cfma(beta[t / per], p[t], z[t]);
}

int dot_chunks(int B, int64_t nalm, int sms) {
  int c = (sms * 4 + B - 1) / B;
  const int64_t maxc = (3 * nalm + 8191) / 8192;
  if (c > maxc) c = int(maxc);
  if (c > 512) c = 512;
  return c < 1 ? 1 : c;
}

int n_sms() {
  static int sms = 0;
  if (sms == 0) {
    int dev = 0, c = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, dev);
    sms = c > 0 ? c : 148;
  }
  return sms;
}

}  // namespace
}  // namespace ps

using namespace ps;

extern "C" int ps_lm_matvec3(const double* S, const double* pre, const double* post, const double* x, double* y,
                             int batch, int64_t nalm, cudaStream_t stream) {
  if (!S || !x || !y || batch < 0 || nalm < 0) return PS_ERR_INVALID;
  if (batch == 0 || nalm == 0) return PS_OK;
  const int64_t total = int64_t(batch) * nalm;
  StatScope sc(PS_K_VECTOR, 36.0 * total, 96.0 * total + 72.0 * nalm, stream);
  const int64_t need = (total + 255) / 256, cap = int64_t(n_sms()) * 8;
  lm_matvec3_kernel<<<int(need < cap ? need : cap), 256, 0, stream>>>(
      S, pre, post, reinterpret_cast<const double2*>(x), reinterpret_cast<double2*>(y), batch, nalm);
  PS_LAUNCH_CHECK();
  return PS_OK;
}

extern "C" int ps_lm_dot_workspace_bytes(int batch, int64_t nalm, size_t* bytes) {
  if (!bytes || batch <= 0 || nalm <= 0) return PS_ERR_INVALID;
  *bytes = sizeof(double) * size_t(batch) * size_t(dot_chunks(batch, nalm, n_sms()));
  return PS_OK;
}

extern "C" int ps_lm_dot(const double* x, const double* y, const double* w, int batch, int64_t nalm, double* out,
                         void* workspace, size_t workspace_bytes, cudaStream_t stream) {
  if (!x || !y || !w || !out || batch <= 0 || nalm <= 0) return PS_ERR_INVALID;
  const int nc = dot_chunks(batch, nalm, n_sms());
  if (!workspace || workspace_bytes < sizeof(double) * size_t(batch) * nc) return PS_ERR_WORKSPACE;
  double* partial = static_cast<double*>(workspace);
  StatScope sc(PS_K_VECTOR, 5.0 * 3 * batch * double(nalm), 32.0 * 3 * batch * double(nalm), stream);
  lm_dot_stage1<<<dim3(nc, batch), DOT_THREADS, 0, stream>>>(reinterpret_cast<const double2*>(x),
                                                             reinterpret_cast<const double2*>(y), w, nalm, nc,
                                                             partial);
  PS_LAUNCH_CHECK();
  lm_dot_stage2<<<(batch + 127) / 128, 128, 0, stream>>>(partial, batch, nc, out);
  PS_LAUNCH_CHECK();
  return PS_OK;
}

extern "C" int ps_lm_matvec3_add(const double* S, const double* x, double* y, int batch, int64_t nalm,
                                 cudaStream_t stream) {
  if (!S || !x || !y || x == y || batch < 0 || nalm < 0) return PS_ERR_INVALID;
  if (batch == 0 || nalm == 0) return PS_OK;
  const int64_t total = int64_t(batch) * nalm;
  StatScope sc(PS_K_VECTOR, 36.0 * total, 144.0 * total + 72.0 * nalm, stream);
  const int64_t need = (total + 255) / 256, cap = int64_t(n_sms()) * 8;
  lm_matvec3_add_kernel<<<int(need < cap ? need : cap), 256, 0, stream>>>(
      S, reinterpret_cast<const double2*>(x), reinterpret_cast<double2*>(y), batch, nalm);
  PS_LAUNCH_CHECK();
  return PS_OK;
}

extern "C" int ps_lm_quad_dot(const double* S, const double* x, const double* w, int batch, int64_t nalm, double* out,
                              void* workspace, size_t workspace_bytes, cudaStream_t stream) {
  if (!S || !x || !w || !out || batch <= 0 || nalm <= 0) return PS_ERR_INVALID;
  const int nc = dot_chunks(batch, nalm, n_sms());
  if (!workspace || workspace_bytes < sizeof(double) * size_t(batch) * nc) return PS_ERR_WORKSPACE;
  double* partial = static_cast<double*>(workspace);
  StatScope sc(PS_K_VECTOR, 40.0 * 3 * batch * double(nalm), 48.0 * batch * double(nalm) + 80.0 * nalm, stream);
  lm_quad_stage1<<<dim3(nc, batch), DOT_THREADS, 0, stream>>>(S, reinterpret_cast<const double2*>(x), w, nalm, nc,
                                                              partial);
  PS_LAUNCH_CHECK();
  lm_dot_stage2<<<(batch + 127) / 128, 128, 0, stream>>>(partial, batch, nc, out);
  PS_LAUNCH_CHECK();
  return PS_OK;
}

extern "C" int ps_cg_xr_update(double* x, const int64_t* slot, const double* alpha, const double* p, double* r,
                               const double* q, int batch, int64_t per, cudaStream_t stream) {
  if (!x || !alpha || !p || !r || !q || batch < 0 || per < 0) return PS_ERR_INVALID;
  if (batch == 0 || per == 0) return PS_OK;
  const int64_t total = int64_t(batch) * per;
  StatScope sc(PS_K_VECTOR, 8.0 * total, 96.0 * total, stream);
  const int64_t need = (total + 255) / 256, cap = int64_t(n_sms()) * 8;
  cg_xr_kernel<<<int(need < cap ? need : cap), 256, 0, stream>>>(
      reinterpret_cast<double2*>(x), slot, alpha, reinterpret_cast<const double2*>(p), reinterpret_cast<double2*>(r),
      reinterpret_cast<const double2*>(q), batch, per);
  PS_LAUNCH_CHECK();
  return PS_OK;
}

extern "C" int ps_cg_direction(double* p, const double* z, const double* beta, int batch, int64_t per,
                               cudaStream_t stream) {
  if (!p || !z || !beta || p == z || batch < 0 || per < 0) return PS_ERR_INVALID;
  if (batch == 0 || per == 0) return PS_OK;
  const int64_t total = int64_t(batch) * per;
  StatScope sc(PS_K_VECTOR, 4.0 * total, 48.0 * total, stream);
  const int64_t need = (total + 255) / 256, cap = int64_t(n_sms()) * 8;
  cg_dir_kernel<<<int(need < cap ? need : cap), 256, 0, stream>>>(reinterpret_cast<double2*>(p),
                                                                  reinterpret_cast<const double2*>(z), beta, batch, per);
  PS_LAUNCH_CHECK();
  return PS_OK;
}
