// Ideal (unit-mask) bispectrum Fisher matrix of BSpecBin (polyspec/bspec_bin.py:
// 699-827) without explicit Wigner 3j symbols, FP64.
//
// The reference sums, per pair of bin triplets with equal sorted bins,
//   Sum_{l1 l2 l3 in the bins} fac tj(l1,l2,l3)^2 Prod_i h_i(l_i) / (4 pi),
// tj = [(l1 l2 l3; -1 -1 2) + (l1 l2 l3; 2 -1 -1) + (l1 l2 l3; -1 2 -1)] / 3, fac = 1 or i
// by the parity of l1 + l2 + l3, and h_i(l) = beam beam' Cinv (2l + 1) per position.  With
// the Gaunt identity of Wigner d-functions (Edmonds 1957, eq. 4.6.2 integrated over two
// Euler angles)
//   Int_{-1}^{1} d^{l1}_{m1 n1} d^{l2}_{m2 n2} d^{l3}_{m3 n3} dx = 2 (l1 l2 l3; m1 m2 m3)(l1 l2 l3; n1 n2 n3),
// tj^2 = (1/18) Sum_{X,Y} Int Prod_i d^{l_i}_{X_i Y_i}, X, Y over the three m-vectors; so the
// l-sum factorises into Gauss-Legendre sums over nodes x_k of products of three binned
// d-sums Phi[g][b][(m, n)][par](x_k) = Sum_{l in b} h_g(l) (+-1)^l d^l_{m n}(x_k), exact when
// the nodes integrate polynomials of degree 3 lmax.  The parity split uses (-1)^(l1+l2+l3) =
// Prod_i (-1)^(l_i).
//
//  * ps_gl_nodes: Gauss-Legendre nodes and weights by Newton iteration on P_n (one thread
//    per node, the three-term recurrence for P_n and P_n').
//  * ps_wigner_binned: Phi for m, n in {-1, 2}: one thread per (node, (m, n), g) runs the
//    upward recurrence
//      l sqrt(((l+1)^2 - m^2)((l+1)^2 - n^2)) d^{l+1} = (2l+1)(l(l+1) x - m n) d^l
//                                                     - (l+1) sqrt((l^2 - m^2)(l^2 - n^2)) d^{l-1}
//    from d^1_{-1,-1} = cos^2(t/2), d^2_{2,2} = cos^4(t/2), d^2_{2,-1} = -2 cos(t/2) sin^3(t/2),
//    d^2_{-1,2} = 2 cos(t/2) sin^3(t/2) (|d| <= 1: no scaling needed) and accumulates the bins.
//  * ps_quad_triple: Sum_k w_k A[ia][k] B[ib][k] C[ic][k] per task (ia, ib, ic): the quadrature of
//    three binned d-sums (TSpecBin's ideal 0- and 2-field terms).
//  * ps_bispec_ideal_contract: per task (three (g, bin) pairs) the two sums
//    S[par] = (1/18) Sum_k w_k Sum_{X,Y} Prod_i Phi[g_i][b_i][(X_i, Y_i)][par](x_k), one CTA per
//    task, the nodes reduced in a fixed order.
#include "ps_common.cuh"
#include "ps_stats.cuh"

namespace ps {
namespace {

__global__ void gl_nodes_kernel(int n, double* __restrict__ x, double* __restrict__ w) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  double z = cos(M_PI * (k + 0.75) / (n + 0.5)), dp = 1.0;
  for (int it = 0; it < 100; ++it) {
    double p0 = 1.0, p1 = z;
    for (int j = 1; j < n; ++j) {
      const double p2 = ((2.0 * j + 1.0) * z * p1 - j * p0) / (j + 1.0);
      p0 = p1;
      p1 = p2;
    }
    dp = n * (z * p1 - p0) / (z * z - 1.0);
    const double dz = p1 / dp;
    z -= dz;
    if (fabs(dz) < 1e-16) break;
  }
  // the derivative at the converged node
  double p0 = 1.0, p1 = z;
  for (int j = 1; j < n; ++j) {
    const double p2 = ((2.0 * j + 1.0) * z * p1 - j * p0) / (j + 1.0);
    p0 = p1;
    p1 = p2;
  }
  dp = n * (z * p1 - p0) / (z * z - 1.0);
  x[k] = z;
  w[k] = 2.0 / ((1.0 - z * z) * dp * dp);
}

// (m, n) of slot q: 0 (-1,-1), 1 (-1,2), 2 (2,-1), 3 (2,2)
__device__ __forceinline__ int slot_m(int q) { return (q & 2) ? 2 : -1; }
__device__ __forceinline__ int slot_n(int q) { return (q & 1) ? 2 : -1; }

__global__ void wigner_binned_kernel(const double* __restrict__ xs, int nk, int lmax, const int* __restrict__ edges,
                                     int nbins, const double* __restrict__ H, int G, double* __restrict__ Phi) {
  const int64_t total = int64_t(G) * 4 * nk;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total; t += int64_t(gridDim.x) * blockDim.x) {
    const int k = int(t % nk);
    const int q = int((t / nk) % 4);
    const int g = int(t / (int64_t(nk) * 4));
    const int m = slot_m(q), n = slot_n(q);
    const double x = xs[k];
    const double c = sqrt(0.5 * (1.0 + x)), s = sqrt(0.5 * (1.0 - x));
    int l0;
    double cur;
    if (q == 0) {
      l0 = 1;
      cur = c * c;
    } else if (q == 3) {
      l0 = 2;
      cur = (c * c) * (c * c);
    } else {
      l0 = 2;
      cur = 2.0 * c * s * s * s * (q == 2 ? -1.0 : 1.0);
    }
    double prev = 0.0;
    const double* h = H + int64_t(g) * (lmax + 1);
    int b = 0;
    double acc0 = 0.0, acc1 = 0.0;
    auto flush = [&](int bb) {
      if (bb >= 0 && bb < nbins) {
        const int64_t o = ((int64_t(g) * nbins + bb) * 4 + q) * 2;
        Phi[o * nk + k] = acc0;
        Phi[(o + 1) * nk + k] = acc1;
      }
      acc0 = 0.0;
      acc1 = 0.0;
    };
    // bins below l0 get zeros
    while (b < nbins && edges[b + 1] <= l0) flush(b++);
    for (int l = l0; l <= lmax; ++l) {
      while (b < nbins && l >= edges[b + 1]) flush(b++);
      if (b >= nbins) break;
      if (l >= edges[b]) {
        const double v = h[l] * cur;
        acc0 += v;
        acc1 += (l & 1) ? -v : v;
      }
      if (l < lmax) {
        const double dl = double(l);
        const double a = (2.0 * dl + 1.0) * (dl * (dl + 1.0) * x - double(m) * n);
        const double bb = (dl + 1.0) * sqrt(fmax(dl * dl - m * m, 0.0) * fmax(dl * dl - n * n, 0.0));
        const double den = dl * sqrt(((dl + 1.0) * (dl + 1.0) - m * m) * ((dl + 1.0) * (dl + 1.0) - n * n));
        const double nxt = (a * cur - bb * prev) / den;
        prev = cur;
        cur = nxt;
      }
    }
    while (b < nbins) flush(b++);
  }
}

__global__ void ideal_contract_kernel(const double* __restrict__ Phi, const double* __restrict__ w, int nk, int G,
                                      int nbins, const int* __restrict__ tasks, double* __restrict__ out) {
  const int task = blockIdx.x;
  const int* tk = tasks + 6 * int64_t(task);
  const int g[3] = {tk[0], tk[2], tk[4]}, bn[3] = {tk[1], tk[3], tk[5]};
  for (int i = 0; i < 3; ++i)
    if (g[i] < 0 || g[i] >= G || bn[i] < 0 || bn[i] >= nbins) {  // a malformed task reads nothing
      if (threadIdx.x == 0) out[2 * int64_t(task)] = out[2 * int64_t(task) + 1] = nan("");
      return;
    }
  // m-vectors X = (-1,-1,2), (2,-1,-1), (-1,2,-1): is position i's entry 2?
  const int two[3][3] = {{0, 0, 1}, {1, 0, 0}, {0, 1, 0}};
  __shared__ double red[2][256];
  double s[2] = {0.0, 0.0};
  for (int k = threadIdx.x; k < nk; k += blockDim.x) {
    const double wk = w[k];
#pragma unroll
    for (int par = 0; par < 2; ++par) {
      double t = 0.0;
      for (int X = 0; X < 3; ++X)
        for (int Y = 0; Y < 3; ++Y) {
          double p = 1.0;
#pragma unroll
          for (int i = 0; i < 3; ++i) {
            const int q = 2 * two[X][i] + two[Y][i];
            p *= Phi[((((int64_t(g[i]) * nbins + bn[i]) * 4 + q) * 2 + par) * nk) + k];
          }
          t += p;
        }
      s[par] += wk * t;
    }
  }
  red[0][threadIdx.x] = s[0];
  red[1][threadIdx.x] = s[1];
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (int(threadIdx.x) < o) {
      red[0][threadIdx.x] += red[0][threadIdx.x + o];
      red[1][threadIdx.x] += red[1][threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[2 * int64_t(task)] = red[0][0] / 18.0;
    out[2 * int64_t(task) + 1] = red[1][0] / 18.0;
  }
}

__global__ void quad_triple_kernel(const double* __restrict__ A, int nA, const double* __restrict__ B, int nB,
                                   const double* __restrict__ C, int nC, const double* __restrict__ w, int nk,
                                   const int* __restrict__ tasks, double* __restrict__ out) {
  const int task = blockIdx.x;
  const int ia = tasks[3 * int64_t(task)], ib = tasks[3 * int64_t(task) + 1], ic = tasks[3 * int64_t(task) + 2];
  if (ia < 0 || ia >= nA || ib < 0 || ib >= nB || ic < 0 || ic >= nC) {  // a malformed task reads nothing
    if (threadIdx.x == 0) out[task] = nan("");
    return;
  }
  const double* a = A + int64_t(ia) * nk;
  const double* b = B + int64_t(ib) * nk;
  const double* c = C + int64_t(ic) * nk;
  __shared__ double red[256];
  double s = 0.0;
  for (int k = threadIdx.x; k < nk; k += blockDim.x) s += w[k] * a[k] * b[k] * c[k];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (int(threadIdx.x) < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[task] = red[0];
}

}  // namespace
}  // namespace ps

using namespace ps;

extern "C" int ps_quad_triple(const double* A, int nA, const double* B, int nB, const double* C, int nC,
                              const double* w, int nk, const int* tasks, int ntask, double* out, cudaStream_t stream) {
  if (!A || !B || !C || !w || !tasks || !out || nA <= 0 || nB <= 0 || nC <= 0 || nk <= 0 || ntask < 0)
    return PS_ERR_INVALID;
  if (ntask == 0) return PS_OK;
  StatScope sc(PS_K_VECTOR, 4.0 * double(ntask) * nk, 32.0 * double(ntask) * nk, stream);
  quad_triple_kernel<<<ntask, 256, 0, stream>>>(A, nA, B, nB, C, nC, w, nk, tasks, out);
  PS_LAUNCH_CHECK();
  return PS_OK;
}

extern "C" int ps_gl_nodes(int n, double* x, double* w, cudaStream_t stream) {
  if (n <= 0 || !x || !w) return PS_ERR_INVALID;
  StatScope sc(PS_K_VECTOR, 0.0, 16.0 * n, stream);
  gl_nodes_kernel<<<(n + 127) / 128, 128, 0, stream>>>(n, x, w);
  PS_LAUNCH_CHECK();
  return PS_OK;
}

extern "C" int ps_wigner_binned(const double* x, int nk, int lmax, const int* edges, int nbins, const double* H, int G,
                                double* Phi, cudaStream_t stream) {
  if (!x || !edges || !H || !Phi || nk <= 0 || lmax < 2 || nbins <= 0 || G <= 0) return PS_ERR_INVALID;
  const int64_t total = int64_t(G) * 4 * nk;
  StatScope sc(PS_K_VECTOR, 12.0 * double(total) * lmax, 8.0 * double(total) * (2 * nbins + lmax), stream);
  int64_t g = (total + 127) / 128;
  if (g > 65535) g = 65535;
  wigner_binned_kernel<<<int(g), 128, 0, stream>>>(x, nk, lmax, edges, nbins, H, G, Phi);
  PS_LAUNCH_CHECK();
  return PS_OK;
}

extern "C" int ps_bispec_ideal_contract(const double* Phi, const double* w, int nk, int G, int nbins, const int* tasks,
                                        int ntask, double* out, cudaStream_t stream) {
  if (!Phi || !w || !tasks || !out || nk <= 0 || G <= 0 || nbins <= 0 || ntask < 0) return PS_ERR_INVALID;
  if (ntask == 0) return PS_OK;
  StatScope sc(PS_K_VECTOR, 2.0 * 9 * 4 * double(ntask) * nk, 8.0 * 3 * 9 * 2 * double(ntask) * nk, stream);
  ideal_contract_kernel<<<ntask, 256, 0, stream>>>(Phi, w, nk, G, nbins, tasks, out);
  PS_LAUNCH_CHECK();
  return PS_OK;
}
