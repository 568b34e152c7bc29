// FP64 ring transforms of the HEALPix SHT: per ring of nphi pixels,
//   synthesis  map_j = sum_{|m| <= mmax} F_m e^{i m (phi0 + 2 pi j / nphi)}   (F_{-m} = F_m^*)
//   adjoint    P_m   = sum_j map_j e^{-i m (phi0 + 2 pi j / nphi)},  m = 0..mmax
// with the HEALPix m-aliasing (m folded modulo nphi).
//
// The two real components of a spin-s map share one complex FFT (their spectra
// are Hermitian): the synthesis transforms conj(c_a) + i conj(c_b) and reads
// map_a, map_b from the real and imaginary parts; the adjoint transforms
// x_a + i x_b and separates X_a = (Z_k + Z*_{N-k})/2, X_b = (Z_k - Z*_{N-k})/(2i).
// A spin-0 map packs a ring with its mirror ring instead (pack = 0; same length
// and phi0; the launch walks the north rings, the equator ring alone): packing two
// different maps would add the rounding of the larger to the smaller at the larger
// one's scale, which shows when batch members differ by many orders of magnitude
// (the Fisher rows of different templates do), while the two rings of one map, or
// the two components of one spin map (mixed by the Legendre stage anyway), share
// their scale.  A CTA runs G such FFTs
// at once (G = 256 / T threads per FFT); the grid is (groups of fields, rings of
// one work length), fields fastest, so that the CTAs of all maps of a ring run
// together and share in L2 the sectors of the ring's phases (stored map-innermost).
// FFTs are radix-2 with stages fused in pairs (one barrier and one shared-memory
// round trip per two stages): decimation in
// frequency for power-of-two rings, Bluestein's chirp-z convolution of
// power-of-two length M >= 2 nphi - 1 for the others.
//
// e^{i m phi0} for the aliases m = k + j nphi of one Fourier index k is
// e^{i k phi0} times a fixed step (+-1 on HEALPix rings, phi0 = pi phi_num / nphi):
// two sincospi per index and field pair instead of one per m and field.
#include "ps_common.cuh"
#include "ps_stats.cuh"

namespace ps {

__device__ __forceinline__ int bitrev(int i, int logn) { return (int)(__brev((unsigned)i) >> (32 - logn)); }
__device__ __forceinline__ int ilog2(int n) { return 31 - __clz(n); }

// e^{i pi q / den} for integer q (exact argument reduction modulo 2 den)
__device__ __forceinline__ double2 expi_pi_ratio(int64_t q, int64_t den) {
  q %= 2 * den;
  if (q < 0) q += 2 * den;
  double s, c;
  sincospi(double(q) / double(den), &s, &c);
  return make_double2(c, s);
}

// twiddle e^{sign 2 pi i j / 2^s} from tw[k] = e^{-2 pi i k / 2^twlog}
__device__ __forceinline__ double2 twid_d(const double2* __restrict__ tw, int j, int s, int twlog, int sign) {
  double2 w = tw[j << (twlog - s)];
  if (sign > 0) w.y = -w.y;
  return w;
}

// Decimation in frequency (natural order in, bit-reversed out) on a[0..2^logn),
// by the T threads with local index u; stages fused in pairs.
__device__ void fft_dif_d(double2* a, int logn, int sign, const double2* __restrict__ tw, int twlog, int u, int T) {
  const int n = 1 << logn;
  int s = logn;
  for (; s >= 2; s -= 2) {
    const int q = 1 << (s - 2);
    for (int t = u; t < n / 4; t += T) {
      const int blk = t >> (s - 2), j = t & (q - 1);
      const int i0 = blk * 4 * q + j, i1 = i0 + q, i2 = i0 + 2 * q, i3 = i0 + 3 * q;
      const double2 x0 = a[i0], x1 = a[i1], x2 = a[i2], x3 = a[i3];
      const double2 y0 = cadd(x0, x2), y2 = cmul(csub(x0, x2), twid_d(tw, j, s, twlog, sign));
      const double2 y1 = cadd(x1, x3), y3 = cmul(csub(x1, x3), twid_d(tw, j + q, s, twlog, sign));
      const double2 w = twid_d(tw, j, s - 1, twlog, sign);
      a[i0] = cadd(y0, y1);
      a[i1] = cmul(csub(y0, y1), w);
      a[i2] = cadd(y2, y3);
      a[i3] = cmul(csub(y2, y3), w);
    }
    __syncthreads();
  }
  if (s == 1) {
    for (int t = u; t < n / 2; t += T) {
      const double2 x0 = a[2 * t], x1 = a[2 * t + 1];
      a[2 * t] = cadd(x0, x1);
      a[2 * t + 1] = csub(x0, x1);
    }
    __syncthreads();
  }
}

// Decimation in time (bit-reversed order in, natural out); stages fused in pairs.
__device__ void fft_dit_d(double2* a, int logn, int sign, const double2* __restrict__ tw, int twlog, int u, int T) {
  const int n = 1 << logn;
  int s = 1;
  if (logn & 1) {
    for (int t = u; t < n / 2; t += T) {
      const double2 x0 = a[2 * t], x1 = a[2 * t + 1];
      a[2 * t] = cadd(x0, x1);
      a[2 * t + 1] = csub(x0, x1);
    }
    __syncthreads();
    s = 2;
  }
  for (; s + 1 <= logn; s += 2) {
    const int q = 1 << (s - 1);
    for (int t = u; t < n / 4; t += T) {
      const int blk = t >> (s - 1), j = t & (q - 1);
      const int i0 = blk * 4 * q + j, i1 = i0 + q, i2 = i0 + 2 * q, i3 = i0 + 3 * q;
      const double2 ws = twid_d(tw, j, s, twlog, sign);
      const double2 v1 = cmul(a[i1], ws), v3 = cmul(a[i3], ws);
      const double2 x0 = a[i0], x2 = a[i2];
      const double2 y0 = cadd(x0, v1), y1 = csub(x0, v1), y2 = cadd(x2, v3), y3 = csub(x2, v3);
      const double2 v2 = cmul(y2, twid_d(tw, j, s + 1, twlog, sign));
      const double2 v3b = cmul(y3, twid_d(tw, j + q, s + 1, twlog, sign));
      a[i0] = cadd(y0, v2);
      a[i2] = csub(y0, v2);
      a[i1] = cadd(y1, v3b);
      a[i3] = csub(y1, v3b);
    }
    __syncthreads();
  }
}

struct RingDFT {
  int N, M, logM;  // M = work length (N for power-of-two rings)
  bool bluestein;
};

__device__ __forceinline__ RingDFT make_dft_d(const RingInfo& g) {
  RingDFT d;
  d.N = g.nphi;
  d.bluestein = g.bs_slot >= 0;
  d.M = d.bluestein ? g.bs_m : d.N;
  d.logM = ilog2(d.M);
  return d;
}

// chirp w_j = e^{-i pi j^2 / N}
__device__ __forceinline__ double2 chirp(int j, int N) {
  const int64_t q = (int64_t(j) * j) % (2 * int64_t(N));
  return expi_pi_ratio(-q, N);
}

// In-place forward DFT (sign -1) of buf[0..N) (natural order); read the
// results with dft_get: bit-reversed for power-of-two N, for Bluestein rings
// M X_k times the chirp factor still to be applied.
__device__ void ring_dft_forward(double2* buf, const RingDFT& d, const double2* __restrict__ tw, int twlog,
                                 const double2* __restrict__ bspec, int u, int T) {
  if (!d.bluestein) {
    fft_dif_d(buf, d.logM, -1, tw, twlog, u, T);
    return;
  }
  for (int j = u; j < d.M; j += T) buf[j] = (j < d.N) ? cmul(buf[j], chirp(j, d.N)) : make_double2(0.0, 0.0);
  __syncthreads();
  fft_dif_d(buf, d.logM, -1, tw, twlog, u, T);
  for (int p = u; p < d.M; p += T) buf[p] = cmul(buf[p], bspec[p]);
  __syncthreads();
  fft_dit_d(buf, d.logM, +1, tw, twlog, u, T);
}

__device__ __forceinline__ double2 dft_get(const double2* buf, const RingDFT& d, int k) {
  if (!d.bluestein) return buf[bitrev(k, d.logM)];
  return cscale(cmul(buf[k], chirp(k, d.N)), 1.0 / double(d.M));
}

// ---------------------------------------------------------------------------
// synthesis: phase [R][mmax+1][nf] -> map [nf][npix]
// grid (ceil(units / G), rings of the class); block T*G threads; smem G*M double2
__global__ void ring_synth_f64(const RingInfo* __restrict__ rings, const int* __restrict__ ring_list, int R,
                               const double2* __restrict__ phase, double* __restrict__ map, int mmax, int nf,
                               int64_t npix, const double2* __restrict__ tw, int twlog,
                               const double2* __restrict__ bs_spec, const int64_t* __restrict__ bs_off, int T,
                               int pack) {
  extern __shared__ double2 dbuf[];
  const int ir = ring_list[blockIdx.y];
  // partner of a packed FFT: the other component of the same map (pack), else the
  // same map on the mirror ring (same nphi and phi0; the list holds north rings)
  const int irb = pack ? ir : R - 1 - ir;
  const RingInfo g = rings[ir];
  const int64_t start_b = rings[irb].start;
  const RingDFT d = make_dft_d(g);
  const double2* bspec = d.bluestein ? bs_spec + bs_off[g.bs_slot] : nullptr;
  const int grp = threadIdx.x / T, u = threadIdx.x - grp * T;
  const int G = blockDim.x / T;
  const int unit = blockIdx.x * G + grp;
  const int fa = pack ? 2 * unit : unit, fb = pack ? fa + 1 : unit;
  const bool va = fa < nf, vb = pack ? fb < nf : (va && irb != ir);
  double2* buf = dbuf + size_t(grp) * d.M;
  const int N = d.N;
  const double2* pha = phase + int64_t(ir) * (mmax + 1) * nf;
  const double2* phb = phase + int64_t(irb) * (mmax + 1) * nf;
  // buf_k = conj(c_a,k) + i conj(c_b,k);  c_k = sum_{m=k mod N} F_m e^{i m phi0} + sum_{m=-k mod N, m>0} conj(...)
  for (int kk = u; kk < N; kk += T) {
    double2 ca = make_double2(0.0, 0.0), cb = ca;
    if (va) {
      // e^{i m phi0} for m = kk + j N is e0 step^j, e0 = e^{i pi phi_num kk / phi_den},
      // step = e^{i pi phi_num N / phi_den} (= +-1 on HEALPix rings, where phi_den = N)
      const double2 e0 = expi_pi_ratio(int64_t(kk) * g.phi_num, g.phi_den);
      const double2 step = expi_pi_ratio(int64_t(N) * g.phi_num, g.phi_den);
      double2 e = e0;
      for (int m = kk; m <= mmax; m += N) {
        ca = cadd(ca, cmul(pha[int64_t(m) * nf + fa], e));
        if (vb) cb = cadd(cb, cmul(phb[int64_t(m) * nf + fb], e));
        e = cmul(e, step);
      }
      // m = m0 + j N with m0 = N - kk (N for kk = 0): e^{i m0 phi0} = conj(e0) step
      e = cmul(cconj(e0), step);
      for (int m = (kk == 0) ? N : N - kk; m <= mmax; m += N) {
        ca = cadd(ca, cconj(cmul(pha[int64_t(m) * nf + fa], e)));
        if (vb) cb = cadd(cb, cconj(cmul(phb[int64_t(m) * nf + fb], e)));
        e = cmul(e, step);
      }
    }
    // a real field keeps only Re(c_0); it must not leak into the partner field of the pair
    if (kk == 0) { ca.y = 0.0; cb.y = 0.0; }
    buf[kk] = make_double2(ca.x + cb.y, -ca.y + cb.x);  // conj(ca) + i conj(cb)
  }
  __syncthreads();
  ring_dft_forward(buf, d, tw, twlog, bspec, u, T);
  if (va) {
    double* oa = map + int64_t(fa) * npix + g.start;
    double* ob = map + int64_t(fb) * npix + start_b;
    for (int j = u; j < N; j += T) {
      const double2 y = dft_get(buf, d, j);
      oa[j] = y.x;
      if (vb) ob[j] = y.y;
    }
  }
}

// adjoint: map [nf][npix] -> phase [R][mmax+1][nf]
__global__ void ring_adjoint_f64(const RingInfo* __restrict__ rings, const int* __restrict__ ring_list, int R,
                                 const double* __restrict__ map, double2* __restrict__ phase, int mmax, int nf,
                                 int64_t npix, const double2* __restrict__ tw, int twlog,
                                 const double2* __restrict__ bs_spec, const int64_t* __restrict__ bs_off, int T,
                               int pack) {
  extern __shared__ double2 dbuf[];
  const int ir = ring_list[blockIdx.y];
  // partner of a packed FFT: the other component of the same map (pack), else the
  // same map on the mirror ring (same nphi and phi0; the list holds north rings)
  const int irb = pack ? ir : R - 1 - ir;
  const RingInfo g = rings[ir];
  const int64_t start_b = rings[irb].start;
  const RingDFT d = make_dft_d(g);
  const double2* bspec = d.bluestein ? bs_spec + bs_off[g.bs_slot] : nullptr;
  const int grp = threadIdx.x / T, u = threadIdx.x - grp * T;
  const int G = blockDim.x / T;
  const int unit = blockIdx.x * G + grp;
  const int fa = pack ? 2 * unit : unit, fb = pack ? fa + 1 : unit;
  const bool va = fa < nf, vb = pack ? fb < nf : (va && irb != ir);
  double2* buf = dbuf + size_t(grp) * d.M;
  const int N = d.N;
  {
    const double* ia = map + int64_t(va ? fa : 0) * npix + g.start;
    const double* ib = map + int64_t(vb ? fb : 0) * npix + (vb ? start_b : g.start);
    for (int j = u; j < N; j += T) buf[j] = make_double2(va ? ia[j] : 0.0, vb ? ib[j] : 0.0);
  }
  __syncthreads();
  ring_dft_forward(buf, d, tw, twlog, bspec, u, T);
  if (va) {
    double2* pha = phase + int64_t(ir) * (mmax + 1) * nf;
    double2* phb = phase + int64_t(irb) * (mmax + 1) * nf;
    for (int k = u; k < N && k <= mmax; k += T) {
      const int k2 = (N - k) % N;
      const double2 z = dft_get(buf, d, k), z2 = cconj(dft_get(buf, d, k2));
      const double2 xa = make_double2(0.5 * (z.x + z2.x), 0.5 * (z.y + z2.y));
      const double2 xb = make_double2(0.5 * (z.y - z2.y), -0.5 * (z.x - z2.x));  // (z - z2) / (2i)
      // e^{-i m phi0} for m = k + j N: e^{-i pi phi_num k / phi_den} conj(step)^j
      double2 e = expi_pi_ratio(-int64_t(k) * g.phi_num, g.phi_den);
      const double2 step = expi_pi_ratio(-int64_t(N) * g.phi_num, g.phi_den);
      for (int m = k; m <= mmax; m += N) {
        pha[int64_t(m) * nf + fa] = cmul(xa, e);
        if (vb) phb[int64_t(m) * nf + fb] = cmul(xb, e);
        e = cmul(e, step);
      }
    }
  }
}

static void fft_shape_d(int work_len, int nf, int pack, int& T, int& G, int& gy) {
  T = std::max(32, std::min(256, work_len / 4));
  G = std::max(1, 256 / T);
  const int units = pack ? (nf + 1) / 2 : nf;
  G = std::min(G, units);
  gy = (units + G - 1) / G;
}

int launch_ring_synth_f64(const Plan& P, const int* d_list, int nrings, int work_len, const double2* phase,
                          double* map, int nf, int pack, cudaStream_t st) {
  if (nrings == 0) return PS_OK;
  int T, G, gy;
  fft_shape_d(work_len, nf, pack, T, G, gy);
  if (nrings > 65535) return PS_ERR_INVALID;
  const size_t smem = size_t(work_len) * G * sizeof(double2);
  if (smem > 48 * 1024) {
    if (cudaFuncSetAttribute(ring_synth_f64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
      return PS_ERR_CUDA;
  }
  int twlog = 0;
  while ((1 << twlog) < P.max_fft) ++twlog;
  StatScope sc(PS_K_FFT_SYNTH, 0.0, 0.0, st);
  ring_synth_f64<<<dim3(gy, nrings), T * G, smem, st>>>(P.d_rings, d_list, P.R, phase, map, P.mmax, nf, P.npix,
                                                         P.d_twiddle, twlog, P.d_bs_spec, P.d_bs_off, T, pack);
  PS_LAUNCH_CHECK();
  return PS_OK;
}

int launch_ring_adjoint_f64(const Plan& P, const int* d_list, int nrings, int work_len, const double* map,
                            double2* phase, int nf, int pack, cudaStream_t st) {
  if (nrings == 0) return PS_OK;
  int T, G, gy;
  fft_shape_d(work_len, nf, pack, T, G, gy);
  if (nrings > 65535) return PS_ERR_INVALID;
  const size_t smem = size_t(work_len) * G * sizeof(double2);
  if (smem > 48 * 1024) {
    if (cudaFuncSetAttribute(ring_adjoint_f64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
      return PS_ERR_CUDA;
  }
  int twlog = 0;
  while ((1 << twlog) < P.max_fft) ++twlog;
  StatScope sc(PS_K_FFT_ADJOINT, 0.0, 0.0, st);
  ring_adjoint_f64<<<dim3(gy, nrings), T * G, smem, st>>>(P.d_rings, d_list, P.R, map, phase, P.mmax, nf, P.npix,
                                                           P.d_twiddle, twlog, P.d_bs_spec, P.d_bs_off, T, pack);
  PS_LAUNCH_CHECK();
  return PS_OK;
}

}  // namespace ps
