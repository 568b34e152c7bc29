// FP64 ring transforms of the HEALPix SHT: per ring of nphi pixels,
//   synthesis  map_j = sum_{|m| <= mmax} F_m e^{i m (phi0 + 2 pi j / nphi)}   (F_{-m} = F_m^*)
//   adjoint    P_m   = sum_j map_j e^{-i m (phi0 + 2 pi j / nphi)},  m = 0..mmax
// with the HEALPix m-aliasing (m folded modulo nphi).  Each CTA owns one ring
// and runs its FFT in shared memory: radix-2 for power-of-two rings (the
// equatorial belt and the cap rings 4i with i a power of two), Bluestein's
// chirp-z convolution of power-of-two length M >= 2 nphi - 1 for the others.
// Rings are launched in classes of equal work length so that each launch
// sizes its shared memory to its class.
#include "ps_common.cuh"
#include "ps_stats.cuh"

namespace ps {

__device__ __forceinline__ int bitrev(int i, int logn) { return (int)(__brev((unsigned)i) >> (32 - logn)); }

// e^{i pi q / den} for integer q (exact argument reduction modulo 2 den)
__device__ __forceinline__ double2 expi_pi_ratio(int64_t q, int64_t den) {
  q %= 2 * den;
  if (q < 0) q += 2 * den;
  double s, c;
  sincospi(double(q) / double(den), &s, &c);
  return make_double2(c, s);
}

// Decimation in frequency, natural order in, bit-reversed order out.
// sign -1: e^{-2 pi i jk/n}.  tw[k] = e^{-2 pi i k / twn}.
__device__ void fft_dif(double2* a, int logn, int sign, const double2* __restrict__ tw, int twlog) {
  const int n = 1 << logn;
  for (int s = logn; s >= 1; --s) {
    const int half = 1 << (s - 1);
    for (int t = threadIdx.x; t < n / 2; t += blockDim.x) {
      const int j = t & (half - 1);
      const int i0 = ((t >> (s - 1)) << s) + j, i1 = i0 + half;
      double2 w = tw[j << (twlog - s)];
      if (sign > 0) w.y = -w.y;
      const double2 u = a[i0], v = a[i1];
      a[i0] = cadd(u, v);
      a[i1] = cmul(csub(u, v), w);
    }
    __syncthreads();
  }
}

// Decimation in time, bit-reversed order in, natural order out.
__device__ void fft_dit(double2* a, int logn, int sign, const double2* __restrict__ tw, int twlog) {
  const int n = 1 << logn;
  for (int s = 1; s <= logn; ++s) {
    const int half = 1 << (s - 1);
    for (int t = threadIdx.x; t < n / 2; t += blockDim.x) {
      const int j = t & (half - 1);
      const int i0 = ((t >> (s - 1)) << s) + j, i1 = i0 + half;
      double2 w = tw[j << (twlog - s)];
      if (sign > 0) w.y = -w.y;
      const double2 u = a[i0], v = cmul(a[i1], w);
      a[i0] = cadd(u, v);
      a[i1] = csub(u, v);
    }
    __syncthreads();
  }
}

__device__ __forceinline__ int ilog2(int n) { return 31 - __clz(n); }

// Forward DFT X_k = sum_j x_j e^{-2 pi i jk/N} of the N values already in
// buf[0..N) (natural order).  On return, get(k) gives X_k.
struct RingDFT {
  int N, M, logM;  // M = work length (N for power-of-two rings)
  bool bluestein;
};

// chirp w_j = e^{-i pi j^2 / N}
__device__ __forceinline__ double2 chirp(int j, int N) {
  const int64_t q = (int64_t(j) * j) % (2 * int64_t(N));
  return expi_pi_ratio(-q, N);
}

// In-place forward DFT of buf[0..N) (natural order) with sign -1.  For
// power-of-two N the result is left in bit-reversed order; for Bluestein
// rings the result X_k * M is left in natural order at buf[k] times the
// chirp factor still to be applied (see dft_get).
__device__ void ring_dft_forward(double2* buf, const RingDFT& d, const double2* __restrict__ tw, int twlog,
                                 const double2* __restrict__ bspec) {
  if (!d.bluestein) {
    fft_dif(buf, d.logM, -1, tw, twlog);
    return;
  }
  for (int j = threadIdx.x; j < d.M; j += blockDim.x) {
    buf[j] = (j < d.N) ? cmul(buf[j], chirp(j, d.N)) : make_double2(0.0, 0.0);
  }
  __syncthreads();
  fft_dif(buf, d.logM, -1, tw, twlog);
  for (int p = threadIdx.x; p < d.M; p += blockDim.x) buf[p] = cmul(buf[p], bspec[p]);
  __syncthreads();
  fft_dit(buf, d.logM, +1, tw, twlog);
}

__device__ __forceinline__ double2 dft_get(const double2* buf, const RingDFT& d, int k) {
  if (!d.bluestein) return buf[bitrev(k, d.logM)];
  return cscale(cmul(buf[k], chirp(k, d.N)), 1.0 / double(d.M));
}

// ---------------------------------------------------------------------------
// synthesis: phase [R][mmax+1][nf] -> map [nf][npix]
__global__ void ring_synth_f64(const RingInfo* __restrict__ rings, const int* __restrict__ ring_list,
                               const double2* __restrict__ phase, double* __restrict__ map, int mmax, int nf,
                               int64_t npix, const double2* __restrict__ tw, int twlog,
                               const double2* __restrict__ bs_spec, const int64_t* __restrict__ bs_off) {
  extern __shared__ double2 buf[];
  const int ir = ring_list[blockIdx.x];
  const RingInfo g = rings[ir];
  RingDFT d;
  d.N = g.nphi;
  d.bluestein = g.bs_slot >= 0;
  d.M = d.bluestein ? g.bs_m : d.N;
  d.logM = ilog2(d.M);
  const double2* bspec = d.bluestein ? bs_spec + bs_off[g.bs_slot] : nullptr;
  const int N = d.N;
  const int64_t pden = g.phi_den;
  for (int f = 0; f < nf; ++f) {
    // c_k = sum_{m = k mod N} F_m e^{i m phi0} + sum_{m = -k mod N, m >= 1} conj(F_m e^{i m phi0});
    // map = Re(DFT_+(c)) = Re(conj(DFT_-(conj(c)))) = Re(DFT_-(conj c)).
    for (int kk = threadIdx.x; kk < N; kk += blockDim.x) {
      double2 c = make_double2(0.0, 0.0);
      for (int m = kk; m <= mmax; m += N) {
        const double2 F = phase[(int64_t(ir) * (mmax + 1) + m) * nf + f];
        c = cadd(c, cmul(F, expi_pi_ratio(int64_t(m) * g.phi_num, pden)));
      }
      for (int m = (kk == 0) ? N : N - kk; m <= mmax; m += N) {
        const double2 F = phase[(int64_t(ir) * (mmax + 1) + m) * nf + f];
        c = cadd(c, cconj(cmul(F, expi_pi_ratio(int64_t(m) * g.phi_num, pden))));
      }
      buf[kk] = cconj(c);
    }
    __syncthreads();
    ring_dft_forward(buf, d, tw, twlog, bspec);
    double* out = map + int64_t(f) * npix + g.start;
    for (int j = threadIdx.x; j < N; j += blockDim.x) out[j] = dft_get(buf, d, j).x;
    __syncthreads();
  }
}

// adjoint: map [nf][npix] -> phase [R][mmax+1][nf]
__global__ void ring_adjoint_f64(const RingInfo* __restrict__ rings, const int* __restrict__ ring_list,
                                 const double* __restrict__ map, double2* __restrict__ phase, int mmax, int nf,
                                 int64_t npix, const double2* __restrict__ tw, int twlog,
                                 const double2* __restrict__ bs_spec, const int64_t* __restrict__ bs_off) {
  extern __shared__ double2 buf[];
  const int ir = ring_list[blockIdx.x];
  const RingInfo g = rings[ir];
  RingDFT d;
  d.N = g.nphi;
  d.bluestein = g.bs_slot >= 0;
  d.M = d.bluestein ? g.bs_m : d.N;
  d.logM = ilog2(d.M);
  const double2* bspec = d.bluestein ? bs_spec + bs_off[g.bs_slot] : nullptr;
  const int N = d.N;
  const int64_t pden = g.phi_den;
  for (int f = 0; f < nf; ++f) {
    const double* in = map + int64_t(f) * npix + g.start;
    for (int j = threadIdx.x; j < N; j += blockDim.x) buf[j] = make_double2(in[j], 0.0);
    __syncthreads();
    ring_dft_forward(buf, d, tw, twlog, bspec);
    for (int m = threadIdx.x; m <= mmax; m += blockDim.x) {
      const double2 X = dft_get(buf, d, m % N);
      phase[(int64_t(ir) * (mmax + 1) + m) * nf + f] = cmul(X, expi_pi_ratio(-int64_t(m) * g.phi_num, pden));
    }
    __syncthreads();
  }
}

int launch_ring_synth_f64(const Plan& P, const int* d_list, int nrings, int work_len, const double2* phase,
                          double* map, int nf, cudaStream_t st) {
  if (nrings == 0) return PS_OK;
  const size_t smem = size_t(work_len) * sizeof(double2);
  const int threads = std::max(32, std::min(256, work_len / 2));
  if (smem > 48 * 1024) {
    if (cudaFuncSetAttribute(ring_synth_f64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
      return PS_ERR_CUDA;
  }
  int twlog = 0;
  while ((1 << twlog) < P.max_fft) ++twlog;
  StatScope sc(PS_K_FFT_SYNTH, 0.0, 0.0, st);
  ring_synth_f64<<<nrings, threads, smem, st>>>(P.d_rings, d_list, phase, map, P.mmax, nf, P.npix, P.d_twiddle,
                                                twlog, P.d_bs_spec, P.d_bs_off);
  PS_LAUNCH_CHECK();
  return PS_OK;
}

int launch_ring_adjoint_f64(const Plan& P, const int* d_list, int nrings, int work_len, const double* map,
                            double2* phase, int nf, cudaStream_t st) {
  if (nrings == 0) return PS_OK;
  const size_t smem = size_t(work_len) * sizeof(double2);
  const int threads = std::max(32, std::min(256, work_len / 2));
  if (smem > 48 * 1024) {
    if (cudaFuncSetAttribute(ring_adjoint_f64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
      return PS_ERR_CUDA;
  }
  int twlog = 0;
  while ((1 << twlog) < P.max_fft) ++twlog;
  StatScope sc(PS_K_FFT_ADJOINT, 0.0, 0.0, st);
  ring_adjoint_f64<<<nrings, threads, smem, st>>>(P.d_rings, d_list, map, phase, P.mmax, nf, P.npix, P.d_twiddle,
                                                  twlog, P.d_bs_spec, P.d_bs_off);
  PS_LAUNCH_CHECK();
  return PS_OK;
}

}  // namespace ps
