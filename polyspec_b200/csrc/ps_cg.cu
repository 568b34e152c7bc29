// Masked conjugate-gradient solve of the optimal S^-1 filter as one C entry
// (ps_cg_solve): the reference's CGD with the harmonic preconditioner
// (polyspec/weighting.py:217-367), batched over independent right-hand sides.
//
// One CG step on the Bn systems still running (vectors [Bn][NF][nalm] complex128):
//   operator   q = B Y^H W Y B p     ps_sht_weighted_roundtrip per spin (mixed plans
//                                    with tables) or ps_synthesis -> weight -> ps_adjoint
//   cg_tail    q += C^-1 p,  partial sums of <p, q>          -> alpha = rz / <p, q>
//   cg_step    x += alpha p, r -= alpha q, z = Sigma r (into q),
//              partial sums of <r, z>                        -> beta, rz, err = rz / rz0
//   cg_dir     p = z + beta p
// where <a, b> = Sum w_m Re(a conj b) with w_m = 1 + (m > 0) (weighting.py:255).  The
// dot products reduce in a fixed order: per-CTA partials, then one thread per system.
// The host reads err after every step (one small copy), records the step count of each
// system, and compacts the systems that continue (err >= tol) to the front of the r and
// p arrays by a gather into the free buffers; x is updated in place at each system's
// original index, so nothing moves at the end.
#include <algorithm>
#include <cmath>
#include <vector>

#include "ps_common.cuh"
#include "ps_stats.cuh"

struct ps_cg {
  const ps_plan* plan;
  int nf;  // 1: T; 3: T, E, B
  int64_t nalm, npix;
  const double* inv_cl;
  const double* sigma;
  const double* beam;
  const double* weight;
  double scale;
  bool fused;   // ps_sht_weighted_roundtrip available for every spin
  double* d_mw;  // m weights [nalm], owned
};

namespace ps {
namespace {

constexpr int CG_THREADS = 256;

size_t al256(size_t x) { return (x + 255) & ~size_t(255); }

__device__ __forceinline__ double block_sum(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  __shared__ double sw[CG_THREADS / 32];
  if ((threadIdx.x & 31) == 0) sw[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int k = 0; k < CG_THREADS / 32; ++k) t += sw[k];
  return t;
}

// grid (nc, Bn): CTA c of system n covers lm indices [c * per, (c + 1) * per).  The
// round-trip result rt may be Q itself (each element is read before it is written).
template <int NF>
__global__ void cg_tail(const double2* rtT, int64_t sT, const double2* rtP, int64_t sP,
                        const double* __restrict__ beam, const double* __restrict__ Cinv,
                        const double2* __restrict__ P, double2* Q, const double* __restrict__ mw,
                        int64_t nalm, double* __restrict__ partial) {
  const int n = blockIdx.y, c = blockIdx.x, nc = gridDim.x;
  const int64_t per = (nalm + nc - 1) / nc, lo = int64_t(c) * per, hi = min(nalm, lo + per);
  const double2* pn = P + int64_t(n) * NF * nalm;
  double2* qn = Q + int64_t(n) * NF * nalm;
  double acc = 0.0;
  for (int64_t i = lo + threadIdx.x; i < hi; i += CG_THREADS) {
    double2 p[NF];
#pragma unroll
    for (int a = 0; a < NF; ++a) p[a] = pn[int64_t(a) * nalm + i];
    double dot = 0.0;
#pragma unroll
    for (int a = 0; a < NF; ++a) {
      double2 q = a == 0 ? rtT[int64_t(n) * sT + i] : rtP[int64_t(n) * sP + int64_t(a - 1) * nalm + i];
      if (beam) q = cscale(q, __ldg(beam + int64_t(a) * nalm + i));
#pragma unroll
      for (int b = 0; b < NF; ++b) q = cfma(__ldg(Cinv + (int64_t(a) * NF + b) * nalm + i), p[b], q);
      qn[int64_t(a) * nalm + i] = q;
      dot += p[a].x * q.x + p[a].y * q.y;
    }
    acc = fma(__ldg(mw + i), dot, acc);
  }
  const double t = block_sum(acc);
  if (threadIdx.x == 0) partial[int64_t(n) * nc + c] = t;
}

// With alpha: x[slot_of[n]] += alpha p, r -= alpha q.  Then z = Sigma r into Q and the
// partial sums of <r, z>.  Without alpha (initialisation): z = Sigma r only.
template <int NF>
__global__ void cg_step(double2* __restrict__ X, const int* __restrict__ orig, const double* __restrict__ alpha,
                        const double2* __restrict__ P, double2* __restrict__ R, double2* __restrict__ Q,
                        const double* __restrict__ Sig, const double* __restrict__ mw, int64_t nalm,
                        double* __restrict__ partial) {
  const int n = blockIdx.y, c = blockIdx.x, nc = gridDim.x;
  const int64_t per = (nalm + nc - 1) / nc, lo = int64_t(c) * per, hi = min(nalm, lo + per);
  const int64_t off = int64_t(n) * NF * nalm;
  const double al = alpha ? alpha[n] : 0.0;
  double2* xn = alpha ? X + int64_t(orig[n]) * NF * nalm : nullptr;
  double acc = 0.0;
  for (int64_t i = lo + threadIdx.x; i < hi; i += CG_THREADS) {
    double2 r[NF];
#pragma unroll
    for (int a = 0; a < NF; ++a) {
      const int64_t k = int64_t(a) * nalm + i;
      r[a] = R[off + k];
      if (alpha) {
        const double2 p = P[off + k], q = Q[off + k];
        xn[k] = cfma(al, p, xn[k]);
        r[a] = cfma(-al, q, r[a]);
        R[off + k] = r[a];
      }
    }
    double dot = 0.0;
#pragma unroll
    for (int a = 0; a < NF; ++a) {
      double2 z = make_double2(0.0, 0.0);
#pragma unroll
      for (int b = 0; b < NF; ++b) z = cfma(__ldg(Sig + (int64_t(a) * NF + b) * nalm + i), r[b], z);
      Q[off + int64_t(a) * nalm + i] = z;
      dot += r[a].x * z.x + r[a].y * z.y;
    }
    acc = fma(__ldg(mw + i), dot, acc);
  }
  const double t = block_sum(acc);
  if (threadIdx.x == 0) partial[int64_t(n) * nc + c] = t;
}

enum { CG_RZ0 = 0, CG_RZ_INIT = 1, CG_ALPHA = 2, CG_NEXT = 3 };

// Per system: sum the partials in order, then the scalar recurrences of one CG step.
// S = [err | rz | rz0 | alpha | beta] each of `cap` doubles.
__global__ void cg_scalars(const double* __restrict__ partial, int nc, int Bn, int mode, int rz0_is_rz,
                           double* __restrict__ S, int cap) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= Bn) return;
  double s = 0.0;
  for (int c = 0; c < nc; ++c) s += partial[int64_t(n) * nc + c];
  double *err = S, *rz = S + cap, *rz0 = S + 2 * cap, *alpha = S + 3 * cap, *beta = S + 4 * cap;
  if (mode == CG_RZ0) {
    rz0[n] = s;
  } else if (mode == CG_RZ_INIT) {
    rz[n] = s;
    if (rz0_is_rz) rz0[n] = s;
    err[n] = rz0[n] != 0.0 ? s / rz0[n] : 0.0;
  } else if (mode == CG_ALPHA) {
    alpha[n] = rz[n] / s;
  } else {
    beta[n] = s / rz[n];
    rz[n] = s;
    err[n] = s / rz0[n];
  }
}

// p = z + beta p over [Bn][per]
__global__ void cg_dir(double2* __restrict__ P, const double2* __restrict__ Z, const double* __restrict__ beta,
                       int Bn, int64_t per) {
  const int64_t total = int64_t(Bn) * per;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total; t += int64_t(gridDim.x) * blockDim.x) {
    const int n = int(t / per);
    P[t] = cfma(beta[n], P[t], Z[t]);
  }
}

// dst = a - b over n elements
__global__ void cg_sub(double2* __restrict__ dst, const double2* __restrict__ a, const double2* __restrict__ b,
                       int64_t n) {
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < n; t += int64_t(gridDim.x) * blockDim.x)
    dst[t] = csub(a[t], b[t]);
}

// dst[k] = src[idx[k]] for k < Bn, rows of `per` elements
__global__ void cg_gather(double2* __restrict__ dst, const double2* __restrict__ src, const int* __restrict__ idx,
                          int Bn, int64_t per) {
  const int64_t total = int64_t(Bn) * per;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total; t += int64_t(gridDim.x) * blockDim.x) {
    const int k = int(t / per);
    dst[t] = src[int64_t(idx[k]) * per + (t - int64_t(k) * per)];
  }
}

// Unfused operator: T0 [Bn][nalm] = beam_T p_T; T2 [Bn][2][nalm] = beam_{E,B} p_{E,B}
__global__ void cg_split_beam(const double2* __restrict__ P, const double* __restrict__ beam, int nf,
                              double2* __restrict__ T0, double2* __restrict__ T2, int Bn, int64_t nalm) {
  const int64_t total = int64_t(Bn) * nf * nalm;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total; t += int64_t(gridDim.x) * blockDim.x) {
    const int64_t i = t % nalm;
    const int a = int((t / nalm) % nf);
    const int n = int(t / (int64_t(nf) * nalm));
    double2 v = P[t];
    if (beam) v = cscale(v, beam[int64_t(a) * nalm + i]);
    if (a == 0)
      T0[int64_t(n) * nalm + i] = v;
    else
      T2[(int64_t(n) * 2 + (a - 1)) * nalm + i] = v;
  }
}

// Unfused operator: maps M0 [Bn][npix] *= w[0], M2 [Bn][2][npix] *= w[1 + c]
__global__ void cg_weight_maps(double* __restrict__ M0, double* __restrict__ M2, const double* __restrict__ w,
                               int nf, int Bn, int64_t npix) {
  const int64_t total = int64_t(Bn) * nf * npix;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total; t += int64_t(gridDim.x) * blockDim.x) {
    const int64_t p = t % npix;
    const int a = int((t / npix) % nf);
    const int n = int(t / (int64_t(nf) * npix));
    const double f = w[int64_t(a) * npix + p];
    if (a == 0)
      M0[int64_t(n) * npix + p] *= f;
    else
      M2[(int64_t(n) * 2 + (a - 1)) * npix + p] *= f;
  }
}

int grid_for(int64_t n) {
  const int64_t need = (n + CG_THREADS - 1) / CG_THREADS, cap = int64_t(device_sms()) * 8;
  return int(std::max<int64_t>(1, std::min(need, cap)));
}

// dot-product chunks per system: about 4 CTAs per SM over the batch, >= 2048 lm each
int cg_chunks(int Bn, int64_t nalm) {
  int64_t c = (int64_t(device_sms()) * 4 + Bn - 1) / Bn;
  c = std::min<int64_t>(c, (nalm + 2047) / 2048);
  c = std::min<int64_t>(c, 1024);
  return int(std::max<int64_t>(c, 1));
}

// workspace layout for up to `cap` systems
struct CgLayout {
  size_t R, P, Q, T, M, sht, partial, scal, idx, total;
};

size_t cg_sht_bytes(const ps_cg* cg, int cap, int* rc) {
  size_t need = 0;
  *rc = PS_OK;
  for (int spin = 0; spin <= (cg->nf == 3 ? 2 : 0); spin += 2) {
    for (int adj = 0; adj < (cg->fused ? 1 : 2); ++adj) {
      size_t b = 0;
      const int r = cg->fused ? ps_roundtrip_workspace_bytes(cg->plan, cap, spin, &b)
                              : ps_sht_workspace_bytes(cg->plan, cap, spin, adj, &b);
      if (r != PS_OK) {
        *rc = r;
        return 0;
      }
      need = std::max(need, b);
    }
  }
  return need;
}

int cg_layout(const ps_cg* cg, int cap, CgLayout& L) {
  const size_t vec = size_t(cap) * cg->nf * size_t(cg->nalm) * sizeof(double2);
  int rc = PS_OK;
  const size_t sht = cg_sht_bytes(cg, cap, &rc);
  if (rc != PS_OK) return rc;
  size_t o = 0;
  L.R = o; o += al256(vec);
  L.P = o; o += al256(vec);
  L.Q = o; o += al256(vec);
  L.T = o; o += cg->fused ? 0 : al256(vec);
  L.M = o; o += cg->fused ? 0 : al256(size_t(cap) * cg->nf * size_t(cg->npix) * sizeof(double));
  L.sht = o; o += al256(std::max<size_t>(sht, 256));
  // Bn * cg_chunks(Bn) <= 4 * sms + Bn
  L.partial = o; o += al256(sizeof(double) * (size_t(device_sms()) * 4 + 2 * size_t(cap)));
  L.scal = o; o += al256(sizeof(double) * 5 * size_t(cap));
  L.idx = o; o += al256(sizeof(int) * 2 * size_t(cap));
  L.total = o;
  return PS_OK;
}

}  // namespace
}  // namespace ps

using namespace ps;

extern "C" int ps_cg_create(const ps_plan* plan, int nfield, const double* inv_cl, const double* sigma,
                            const double* beam, const double* weight, double scale, ps_cg** out) {
  if (!out) return PS_ERR_INVALID;
  *out = nullptr;
  if (!plan || (nfield != 1 && nfield != 3) || !inv_cl || !sigma || !weight) return PS_ERR_INVALID;
  int nside = 0, lmax = 0;
  int64_t npix = 0, nalm = 0;
  int rc = ps_plan_info(plan, &nside, &lmax, &npix, &nalm);
  if (rc != PS_OK) return rc;
  // the plan's orders: nalm = Sum_{m <= mmax} (lmax + 1 - m)
  std::vector<double> mw(static_cast<size_t>(nalm));
  {
    int64_t i = 0;
    for (int m = 0; m <= lmax && i < nalm; ++m)
      for (int l = m; l <= lmax && i < nalm; ++l) mw[size_t(i++)] = m > 0 ? 2.0 : 1.0;
    if (i != nalm) return PS_ERR_INVALID;
  }
  ps_cg* cg = new ps_cg();
  cg->plan = plan;
  cg->nf = nfield;
  cg->nalm = nalm;
  cg->npix = npix;
  cg->inv_cl = inv_cl;
  cg->sigma = sigma;
  cg->beam = beam;
  cg->weight = weight;
  cg->scale = scale;
  size_t probe = 0;
  if (nfield == 3 && ps_sht_workspace_bytes(plan, 1, 2, 0, &probe) != PS_OK) {
    delete cg;
    return PS_ERR_INVALID;  // the plan has no spin-2 transforms
  }
  cg->fused = ps_roundtrip_workspace_bytes(plan, 1, 0, &probe) == PS_OK &&
              (nfield == 1 || ps_roundtrip_workspace_bytes(plan, 1, 2, &probe) == PS_OK);
  if (cudaMalloc(&cg->d_mw, sizeof(double) * size_t(nalm)) != cudaSuccess) {
    delete cg;
    return PS_ERR_NOMEM;
  }
  if (cudaMemcpy(cg->d_mw, mw.data(), sizeof(double) * size_t(nalm), cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaFree(cg->d_mw);
    delete cg;
    return PS_ERR_CUDA;
  }
  *out = cg;
  return PS_OK;
}

extern "C" int ps_cg_destroy(ps_cg* cg) {
  if (!cg) return PS_ERR_INVALID;
  cudaFree(cg->d_mw);
  delete cg;
  return PS_OK;
}

extern "C" int ps_cg_workspace_bytes(const ps_cg* cg, int batch, size_t* bytes) {
  if (!cg || !bytes || batch <= 0) return PS_ERR_INVALID;
  CgLayout L;
  const int rc = cg_layout(cg, batch, L);
  if (rc != PS_OK) return rc;
  *bytes = L.total;
  return PS_OK;
}

namespace {

// q = B Y^H W Y B p + C^-1 p for the first Bn systems of P, partial sums of <p, q>
int cg_apply(const ps_cg* cg, const CgLayout& L, char* ws, size_t ws_sht_bytes, const double2* P, double2* Q,
             int Bn, double* partial, int nc, cudaStream_t st) {
  const int64_t nalm = cg->nalm, npix = cg->npix;
  const int nf = cg->nf;
  const double2 *rtT, *rtP;
  int64_t sT, sP;
  const double* tail_beam;
  if (cg->fused) {
    for (int spin = 0; spin <= (nf == 3 ? 2 : 0); spin += 2) {
      const int c0 = spin ? 1 : 0;
      const int rc = ps_sht_weighted_roundtrip(
          cg->plan, reinterpret_cast<const double*>(P + c0 * nalm), reinterpret_cast<double*>(Q + c0 * nalm),
          int64_t(nf) * nalm, Bn, spin, cg->weight + c0 * npix, cg->beam ? cg->beam + c0 * nalm : nullptr, cg->scale,
          ws + L.sht, ws_sht_bytes, st);
      if (rc != PS_OK) return rc;
    }
    rtT = Q;
    rtP = Q + nalm;
    sT = sP = int64_t(nf) * nalm;
    tail_beam = nullptr;
  } else {
    double2* T0 = reinterpret_cast<double2*>(ws + L.T);
    double2* T2 = T0 + int64_t(Bn) * nalm;
    double* M0 = reinterpret_cast<double*>(ws + L.M);
    double* M2 = M0 + int64_t(Bn) * npix;
    {
      StatScope sc(PS_K_VECTOR, 0.0, 32.0 * Bn * nf * double(nalm), st);
      cg_split_beam<<<grid_for(int64_t(Bn) * nf * nalm), CG_THREADS, 0, st>>>(P, cg->beam, nf, T0, T2, Bn, nalm);
      PS_LAUNCH_CHECK();
    }
    int rc = ps_synthesis(cg->plan, reinterpret_cast<const double*>(T0), M0, Bn, 0, ws + L.sht, ws_sht_bytes, st);
    if (rc == PS_OK && nf == 3)
      rc = ps_synthesis(cg->plan, reinterpret_cast<const double*>(T2), M2, Bn, 2, ws + L.sht, ws_sht_bytes, st);
    if (rc != PS_OK) return rc;
    {
      StatScope sc(PS_K_PIXEL, double(Bn) * nf * npix, 24.0 * Bn * nf * double(npix), st);
      cg_weight_maps<<<grid_for(int64_t(Bn) * nf * npix), CG_THREADS, 0, st>>>(M0, M2, cg->weight, nf, Bn, npix);
      PS_LAUNCH_CHECK();
    }
    rc = ps_adjoint(cg->plan, M0, reinterpret_cast<double*>(T0), Bn, 0, cg->scale, ws + L.sht, ws_sht_bytes, st);
    if (rc == PS_OK && nf == 3)
      rc = ps_adjoint(cg->plan, M2, reinterpret_cast<double*>(T2), Bn, 2, cg->scale, ws + L.sht, ws_sht_bytes, st);
    if (rc != PS_OK) return rc;
    rtT = T0;
    rtP = T2;
    sT = nalm;
    sP = 2 * nalm;
    tail_beam = cg->beam;
  }
  StatScope sc(PS_K_VECTOR, 40.0 * Bn * nf * double(nalm), 48.0 * Bn * nf * double(nalm) + 8.0 * nf * nf * nalm, st);
  if (nf == 3)
    cg_tail<3><<<dim3(nc, Bn), CG_THREADS, 0, st>>>(rtT, sT, rtP, sP, tail_beam, cg->inv_cl, P, Q, cg->d_mw, nalm,
                                                     partial);
  else
    cg_tail<1><<<dim3(nc, Bn), CG_THREADS, 0, st>>>(rtT, sT, rtP, sP, tail_beam, cg->inv_cl, P, Q, cg->d_mw, nalm,
                                                     partial);
  PS_LAUNCH_CHECK();
  return PS_OK;
}

int cg_precond(const ps_cg* cg, double2* X, const int* orig, const double* alpha, const double2* P, double2* R,
               double2* Q, int Bn, double* partial, int nc, cudaStream_t st) {
  const int64_t nalm = cg->nalm;
  StatScope sc(PS_K_VECTOR, 40.0 * Bn * cg->nf * double(nalm),
               (alpha ? 96.0 : 32.0) * Bn * cg->nf * double(nalm) + 8.0 * cg->nf * cg->nf * nalm, st);
  if (cg->nf == 3)
    cg_step<3><<<dim3(nc, Bn), CG_THREADS, 0, st>>>(X, orig, alpha, P, R, Q, cg->sigma, cg->d_mw, nalm, partial);
  else
    cg_step<1><<<dim3(nc, Bn), CG_THREADS, 0, st>>>(X, orig, alpha, P, R, Q, cg->sigma, cg->d_mw, nalm, partial);
  PS_LAUNCH_CHECK();
  return PS_OK;
}

int cg_reduce(const double* partial, int nc, int Bn, int mode, int rz0_is_rz, double* S, int cap, cudaStream_t st) {
  cg_scalars<<<(Bn + 127) / 128, 128, 0, st>>>(partial, nc, Bn, mode, rz0_is_rz, S, cap);
  PS_LAUNCH_CHECK();
  return PS_OK;
}

}  // namespace

#define CG_TRY(x)                 \
  do {                            \
    const int _rc = (x);          \
    if (_rc != PS_OK) return _rc; \
  } while (0)
#define CG_CUDA(x)                                  \
  do {                                              \
    if ((x) != cudaSuccess) return PS_ERR_CUDA;     \
  } while (0)

extern "C" int ps_cg_solve(ps_cg* cg, const double* b, const double* x0, double* x, int batch, int max_iter,
                           double tol, int* iters, double* final_err, void* workspace, size_t workspace_bytes,
                           cudaStream_t stream) {
  if (!cg || !b || !x || batch < 0 || max_iter < 0 || !(tol >= 0.0)) return PS_ERR_INVALID;
  if (batch == 0) return PS_OK;
  CgLayout L;
  CG_TRY(cg_layout(cg, batch, L));
  if (!workspace || workspace_bytes < L.total) return PS_ERR_WORKSPACE;
  const int cap = batch, nf = cg->nf;
  const int64_t nalm = cg->nalm, per = int64_t(nf) * nalm;
  const size_t vec_bytes = size_t(batch) * size_t(per) * sizeof(double2);
  char* ws = static_cast<char*>(workspace);
  double2* R = reinterpret_cast<double2*>(ws + L.R);
  double2* P = reinterpret_cast<double2*>(ws + L.P);
  double2* Q = reinterpret_cast<double2*>(ws + L.Q);
  double* partial = reinterpret_cast<double*>(ws + L.partial);
  double* S = reinterpret_cast<double*>(ws + L.scal);
  int* d_orig = reinterpret_cast<int*>(ws + L.idx);
  int* d_gidx = d_orig + cap;
  const size_t sht_bytes = L.partial - L.sht;
  double2* X = reinterpret_cast<double2*>(x);
  const double2* Bv = reinterpret_cast<const double2*>(b);

  std::vector<int> orig(static_cast<size_t>(batch)), gidx;
  for (int n = 0; n < batch; ++n) orig[size_t(n)] = n;
  std::vector<double> host(5 * static_cast<size_t>(cap));
  std::vector<int> it_count(static_cast<size_t>(batch), 0);
  std::vector<double> err_out(static_cast<size_t>(batch), 0.0);
  CG_CUDA(cudaMemcpyAsync(d_orig, orig.data(), sizeof(int) * batch, cudaMemcpyHostToDevice, stream));

  // r = b - A x0 (x = x0) or r = b (x = 0); z = M r; rz = <r, z>; rz0 = <b, M b>; p = z
  int nc = cg_chunks(batch, nalm);
  if (x0) {
    CG_TRY(cg_precond(cg, nullptr, nullptr, nullptr, nullptr, const_cast<double2*>(Bv), Q, batch, partial, nc,
                      stream));
    CG_TRY(cg_reduce(partial, nc, batch, CG_RZ0, 0, S, cap, stream));
    if (x0 != x) CG_CUDA(cudaMemcpyAsync(x, x0, vec_bytes, cudaMemcpyDeviceToDevice, stream));
    CG_CUDA(cudaMemcpyAsync(P, x0, vec_bytes, cudaMemcpyDeviceToDevice, stream));
    CG_TRY(cg_apply(cg, L, ws, sht_bytes, P, Q, batch, partial, nc, stream));
    cg_sub<<<grid_for(int64_t(batch) * per), CG_THREADS, 0, stream>>>(R, Bv, Q, int64_t(batch) * per);
    PS_LAUNCH_CHECK();
  } else {
    CG_CUDA(cudaMemsetAsync(x, 0, vec_bytes, stream));
    CG_CUDA(cudaMemcpyAsync(R, b, vec_bytes, cudaMemcpyDeviceToDevice, stream));
  }
  CG_TRY(cg_precond(cg, nullptr, nullptr, nullptr, nullptr, R, Q, batch, partial, nc, stream));
  CG_TRY(cg_reduce(partial, nc, batch, CG_RZ_INIT, x0 ? 0 : 1, S, cap, stream));
  CG_CUDA(cudaMemcpyAsync(P, Q, vec_bytes, cudaMemcpyDeviceToDevice, stream));

  // systems with b^T M b = 0 are solved at step 0
  CG_CUDA(cudaMemcpyAsync(host.data(), S, sizeof(double) * 3 * cap, cudaMemcpyDeviceToHost, stream));
  CG_CUDA(cudaStreamSynchronize(stream));
  int Bn = 0;
  gidx.clear();
  for (int n = 0; n < batch; ++n) {
    if (host[size_t(2 * cap + n)] == 0.0) continue;
    gidx.push_back(n);
  }
  auto compact = [&](int Bnew) -> int {
    // keep the systems listed in gidx (slots, ascending): gather r and p into the free buffers
    if (Bnew == 0) return PS_OK;
    CG_CUDA(cudaMemcpyAsync(d_gidx, gidx.data(), sizeof(int) * Bnew, cudaMemcpyHostToDevice, stream));
    cg_gather<<<grid_for(int64_t(Bnew) * per), CG_THREADS, 0, stream>>>(Q, P, d_gidx, Bnew, per);
    PS_LAUNCH_CHECK();
    std::swap(P, Q);
    cg_gather<<<grid_for(int64_t(Bnew) * per), CG_THREADS, 0, stream>>>(Q, R, d_gidx, Bnew, per);
    PS_LAUNCH_CHECK();
    std::swap(R, Q);
    std::vector<double> s2(5 * size_t(cap), 0.0);
    std::vector<int> o2(static_cast<size_t>(Bnew));
    for (int k = 0; k < Bnew; ++k) {
      const int j = gidx[size_t(k)];
      for (int f = 0; f < 3; ++f) s2[size_t(f * cap + k)] = host[size_t(f * cap + j)];
      o2[size_t(k)] = orig[size_t(j)];
    }
    orig.assign(o2.begin(), o2.end());
    host.swap(s2);
    CG_CUDA(cudaMemcpyAsync(S, host.data(), sizeof(double) * 3 * cap, cudaMemcpyHostToDevice, stream));
    CG_CUDA(cudaMemcpyAsync(d_orig, orig.data(), sizeof(int) * Bnew, cudaMemcpyHostToDevice, stream));
    // the host buffers are reused after the next synchronisation only
    return PS_OK;
  };
  Bn = int(gidx.size());
  if (Bn < batch) CG_TRY(compact(Bn));

  for (int step = 1; step <= max_iter && Bn > 0; ++step) {
    nc = cg_chunks(Bn, nalm);
    CG_TRY(cg_apply(cg, L, ws, sht_bytes, P, Q, Bn, partial, nc, stream));
    CG_TRY(cg_reduce(partial, nc, Bn, CG_ALPHA, 0, S, cap, stream));
    CG_TRY(cg_precond(cg, X, d_orig, S + 3 * cap, P, R, Q, Bn, partial, nc, stream));
    CG_TRY(cg_reduce(partial, nc, Bn, CG_NEXT, 0, S, cap, stream));
    {
      StatScope sc(PS_K_VECTOR, 2.0 * Bn * double(per), 48.0 * Bn * double(per), stream);
      cg_dir<<<grid_for(int64_t(Bn) * per), CG_THREADS, 0, stream>>>(P, Q, S + 4 * cap, Bn, per);
      PS_LAUNCH_CHECK();
    }
    CG_CUDA(cudaMemcpyAsync(host.data(), S, sizeof(double) * 3 * cap, cudaMemcpyDeviceToHost, stream));
    CG_CUDA(cudaStreamSynchronize(stream));
    gidx.clear();
    for (int k = 0; k < Bn; ++k) {
      const int n = orig[size_t(k)];
      const double e = host[size_t(k)];
      it_count[size_t(n)] = step;
      err_out[size_t(n)] = e;
      if (!(e < tol)) gidx.push_back(k);  // a NaN error keeps running, as in the reference
    }
    const int Bnew = int(gidx.size());
    if (Bnew < Bn) CG_TRY(compact(Bnew));
    Bn = Bnew;
  }
  CG_CUDA(cudaStreamSynchronize(stream));
  if (iters)
    for (int n = 0; n < batch; ++n) iters[n] = it_count[size_t(n)];
  if (final_err)
    for (int n = 0; n < batch; ++n) final_err[n] = err_out[size_t(n)];
  return Bn > 0 ? PS_ERR_NOT_CONVERGED : PS_OK;
}
