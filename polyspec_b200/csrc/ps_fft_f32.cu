// FP32 ring transforms of the mixed-precision HEALPix SHT (maps stay FP64 in
// HBM; the per-ring phases and the FFTs run in FP32).  Per ring of nphi pixels:
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
// at once (G = 256 / T threads per FFT), so small rings keep every thread busy; the
// grid is (groups of fields, rings of one work length), fields fastest, so that the
// CTAs of all maps of a ring run together and share in L2 the sectors of the ring's
// phases (stored map-innermost).
// FFTs are radix-2 with stages fused in threes (one barrier and one shared-memory
// round trip per three stages): decimation in frequency for power-of-two rings,
// Bluestein's chirp-z convolution of power-of-two length M >= 2 nphi - 1 for the
// others.  Rings are launched in classes of equal work length.  The ring rotations
// e^{i m phi0} and the Bluestein chirps come from tables of the plan (computed in FP64
// on the host), so no kernel evaluates a sine or cosine.
#include "ps_common.cuh"
#include "ps_stats.cuh"

namespace ps {

__device__ __forceinline__ float2 fadd2(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 fsub2(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 fmul2(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 fconj2(float2 a) { return make_float2(a.x, -a.y); }

__device__ __forceinline__ int bitrev_f(int i, int logn) { return (int)(__brev((unsigned)i) >> (32 - logn)); }
__device__ __forceinline__ int ilog2_f(int n) { return 31 - __clz(n); }


// twiddle e^{sign 2 pi i j / 2^s} from tw[k] = e^{-2 pi i k / 2^twlog}
__device__ __forceinline__ float2 twid(const float2* __restrict__ tw, int j, int s, int twlog, int sign) {
  float2 w = tw[j << (twlog - s)];
  if (sign > 0) w.y = -w.y;
  return w;
}

// Decimation in frequency (natural order in, bit-reversed out) on a[0..2^logn), by the T threads
// with local index u; stages fused in threes (one barrier and one shared-memory round trip per
// three radix-2 stages, the eight points of a butterfly group in registers), the last one or two
// stages as one radix-2 or radix-4 pass.
__device__ void fft_dif_f(float2* a, int logn, int sign, const float2* __restrict__ tw, int twlog, int u, int T) {
  const int n = 1 << logn;
  int s = logn;
  for (; s >= 3; s -= 3) {
    const int q = 1 << (s - 3);
    for (int t = u; t < n / 8; t += T) {
      const int blk = t >> (s - 3), j = t & (q - 1);
      const int i0 = blk * 8 * q + j;
      float2 x[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) x[k] = a[i0 + k * q];
#pragma unroll
      for (int k = 0; k < 4; ++k) {  // stage s: pairs (k, k + 4)
        const float2 d = fsub2(x[k], x[k + 4]);
        x[k] = fadd2(x[k], x[k + 4]);
        x[k + 4] = fmul2(d, twid(tw, j + k * q, s, twlog, sign));
      }
      const float2 w0 = twid(tw, j, s - 1, twlog, sign), w1 = twid(tw, j + q, s - 1, twlog, sign);
#pragma unroll
      for (int h = 0; h < 8; h += 4) {  // stage s - 1: pairs (k, k + 2) of each half
#pragma unroll
        for (int k = 0; k < 2; ++k) {
          const float2 d = fsub2(x[h + k], x[h + k + 2]);
          x[h + k] = fadd2(x[h + k], x[h + k + 2]);
          x[h + k + 2] = fmul2(d, k ? w1 : w0);
        }
      }
      const float2 w2 = twid(tw, j, s - 2, twlog, sign);
#pragma unroll
      for (int k = 0; k < 8; k += 2) {  // stage s - 2: pairs (k, k + 1)
        const float2 d = fsub2(x[k], x[k + 1]);
        x[k] = fadd2(x[k], x[k + 1]);
        x[k + 1] = fmul2(d, w2);
      }
#pragma unroll
      for (int k = 0; k < 8; ++k) a[i0 + k * q] = x[k];
    }
    __syncthreads();
  }
  if (s == 2) {
    for (int t = u; t < n / 4; t += T) {
      const int i0 = 4 * t;
      const float2 x0 = a[i0], x1 = a[i0 + 1], x2 = a[i0 + 2], x3 = a[i0 + 3];
      const float2 y0 = fadd2(x0, x2), y2 = fmul2(fsub2(x0, x2), twid(tw, 0, 2, twlog, sign));
      const float2 y1 = fadd2(x1, x3), y3 = fmul2(fsub2(x1, x3), twid(tw, 1, 2, twlog, sign));
      const float2 w = twid(tw, 0, 1, twlog, sign);
      a[i0] = fadd2(y0, y1);
      a[i0 + 1] = fmul2(fsub2(y0, y1), w);
      a[i0 + 2] = fadd2(y2, y3);
      a[i0 + 3] = fmul2(fsub2(y2, y3), w);
    }
    __syncthreads();
  } else if (s == 1) {
    for (int t = u; t < n / 2; t += T) {
      const float2 x0 = a[2 * t], x1 = a[2 * t + 1];
      a[2 * t] = fadd2(x0, x1);
      a[2 * t + 1] = fsub2(x0, x1);
    }
    __syncthreads();
  }
}

// Decimation in time (bit-reversed order in, natural out): the first one or two stages as one
// radix-2 or radix-4 pass, then stages fused in threes.
__device__ void fft_dit_f(float2* a, int logn, int sign, const float2* __restrict__ tw, int twlog, int u, int T) {
  const int n = 1 << logn;
  int s = 1;
  if (logn % 3 == 1) {
    for (int t = u; t < n / 2; t += T) {
      const float2 x0 = a[2 * t], x1 = a[2 * t + 1];
      a[2 * t] = fadd2(x0, x1);
      a[2 * t + 1] = fsub2(x0, x1);
    }
    __syncthreads();
    s = 2;
  } else if (logn % 3 == 2) {
    for (int t = u; t < n / 4; t += T) {
      const int i0 = 4 * t;
      const float2 ws = twid(tw, 0, 1, twlog, sign);
      const float2 v1 = fmul2(a[i0 + 1], ws), v3 = fmul2(a[i0 + 3], ws);
      const float2 x0 = a[i0], x2 = a[i0 + 2];
      const float2 y0 = fadd2(x0, v1), y1 = fsub2(x0, v1), y2 = fadd2(x2, v3), y3 = fsub2(x2, v3);
      const float2 v2 = fmul2(y2, twid(tw, 0, 2, twlog, sign));
      const float2 v3b = fmul2(y3, twid(tw, 1, 2, twlog, sign));
      a[i0] = fadd2(y0, v2);
      a[i0 + 2] = fsub2(y0, v2);
      a[i0 + 1] = fadd2(y1, v3b);
      a[i0 + 3] = fsub2(y1, v3b);
    }
    __syncthreads();
    s = 3;
  }
  for (; s + 2 <= logn; s += 3) {
    const int q = 1 << (s - 1);
    for (int t = u; t < n / 8; t += T) {
      const int blk = t >> (s - 1), j = t & (q - 1);
      const int i0 = blk * 8 * q + j;
      float2 x[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) x[k] = a[i0 + k * q];
      const float2 w0 = twid(tw, j, s, twlog, sign);
#pragma unroll
      for (int k = 0; k < 8; k += 2) {  // stage s: pairs (k, k + 1)
        const float2 v = fmul2(x[k + 1], w0);
        x[k + 1] = fsub2(x[k], v);
        x[k] = fadd2(x[k], v);
      }
      const float2 w1a = twid(tw, j, s + 1, twlog, sign), w1b = twid(tw, j + q, s + 1, twlog, sign);
#pragma unroll
      for (int h = 0; h < 8; h += 4) {  // stage s + 1: pairs (k, k + 2) of each half
#pragma unroll
        for (int k = 0; k < 2; ++k) {
          const float2 v = fmul2(x[h + k + 2], k ? w1b : w1a);
          x[h + k + 2] = fsub2(x[h + k], v);
          x[h + k] = fadd2(x[h + k], v);
        }
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) {  // stage s + 2: pairs (k, k + 4)
        const float2 v = fmul2(x[k + 4], twid(tw, j + k * q, s + 2, twlog, sign));
        x[k + 4] = fsub2(x[k], v);
        x[k] = fadd2(x[k], v);
      }
#pragma unroll
      for (int k = 0; k < 8; ++k) a[i0 + k * q] = x[k];
    }
    __syncthreads();
  }
}

struct RingDFTf {
  int N, M, logM;
  bool bluestein;
  const float2* chirp;  // e^{-i pi j^2 / N}, j < N (the plan's table of this ring length)
};

// In-place forward DFT (sign -1) of buf[0..N); read results with dft_get_f.
__device__ void ring_dft_forward_f(float2* buf, const RingDFTf& d, const float2* __restrict__ tw, int twlog,
                                   const float2* __restrict__ bspec, int u, int T) {
  if (!d.bluestein) {
    fft_dif_f(buf, d.logM, -1, tw, twlog, u, T);
    return;
  }
  for (int j = u; j < d.M; j += T) buf[j] = (j < d.N) ? fmul2(buf[j], d.chirp[j]) : make_float2(0.f, 0.f);
  __syncthreads();
  fft_dif_f(buf, d.logM, -1, tw, twlog, u, T);
  for (int p = u; p < d.M; p += T) buf[p] = fmul2(buf[p], bspec[p]);
  __syncthreads();
  fft_dit_f(buf, d.logM, +1, tw, twlog, u, T);
}

__device__ __forceinline__ float2 dft_get_f(const float2* buf, const RingDFTf& d, int k) {
  if (!d.bluestein) return buf[bitrev_f(k, d.logM)];
  const float2 v = fmul2(buf[k], d.chirp[k]);
  const float s = 1.0f / float(d.M);
  return make_float2(v.x * s, v.y * s);
}

__device__ __forceinline__ RingDFTf make_dft(const RingInfo& g, const float2* __restrict__ chirp,
                                             const int64_t* __restrict__ chirp_off) {
  RingDFTf d;
  d.N = g.nphi;
  d.bluestein = g.bs_slot >= 0;
  d.M = d.bluestein ? g.bs_m : d.N;
  d.logM = ilog2_f(d.M);
  d.chirp = d.bluestein ? chirp + chirp_off[g.bs_slot] : nullptr;
  return d;
}

// ---------------------------------------------------------------------------
// synthesis: phase [R][mmax+1][nf] (complex64) -> map [nf][npix] (float64)
// grid (ceil(units / G), rings of the class); block T*G threads; smem G*M float2
__global__ void ring_synth_f32(const RingInfo* __restrict__ rings, const int* __restrict__ ring_list, int R,
                               const float2* __restrict__ phase, double* __restrict__ map, int mmax, int nf,
                               int64_t npix, const float2* __restrict__ tw, int twlog,
                               const float2* __restrict__ bs_spec, const int64_t* __restrict__ bs_off,
                               const float2* __restrict__ rot, const float2* __restrict__ chirp,
                               const int64_t* __restrict__ chirp_off, int T, int pack) {
  extern __shared__ float2 fbuf[];
  const int ir = ring_list[blockIdx.y];
  // partner of a packed FFT: the other component of the same map (pack), else the
  // same map on the mirror ring (same nphi and phi0; the list holds north rings)
  const int irb = pack ? ir : R - 1 - ir;
  const RingInfo g = rings[ir];
  const int64_t start_b = rings[irb].start;
  const RingDFTf d = make_dft(g, chirp, chirp_off);
  const float2* rotr = rot + int64_t(min(ir, R - 1 - ir)) * (mmax + 1);  // e^{i m phi0} of this ring
  const float2* bspec = d.bluestein ? bs_spec + bs_off[g.bs_slot] : nullptr;
  const int grp = threadIdx.x / T, u = threadIdx.x - grp * T;
  const int G = blockDim.x / T;
  const int unit = blockIdx.x * G + grp;
  const int fa = pack ? 2 * unit : unit, fb = pack ? fa + 1 : unit;
  const bool va = fa < nf, vb = pack ? fb < nf : (va && irb != ir);
  float2* buf = fbuf + size_t(grp) * d.M;
  const int N = d.N;
  const float2* pha = phase + int64_t(ir) * (mmax + 1) * nf;
  const float2* phb = phase + int64_t(irb) * (mmax + 1) * nf;
  // buf_k = conj(c_a,k) + i conj(c_b,k);  c_k = sum_{m=k mod N} F_m e^{i m phi0} + sum_{m=-k mod N, m>0} conj(...)
  for (int kk = u; kk < N; kk += T) {
    float2 ca = make_float2(0.f, 0.f), cb = ca;
    if (va) {
      for (int m = kk; m <= mmax; m += N) {
        const float2 e = rotr[m];
        ca = fadd2(ca, fmul2(pha[int64_t(m) * nf + fa], e));
        if (vb) cb = fadd2(cb, fmul2(phb[int64_t(m) * nf + fb], e));
      }
      for (int m = (kk == 0) ? N : N - kk; m <= mmax; m += N) {
        const float2 e = rotr[m];
        ca = fadd2(ca, fconj2(fmul2(pha[int64_t(m) * nf + fa], e)));
        if (vb) cb = fadd2(cb, fconj2(fmul2(phb[int64_t(m) * nf + fb], e)));
      }
    }
    // a real field keeps only Re(c_0) (F_0's imaginary part drops out of the
    // real map); it must not leak into the partner field of the packed pair
    if (kk == 0) { ca.y = 0.f; cb.y = 0.f; }
    // conj(ca) + i conj(cb)
    buf[kk] = make_float2(ca.x + cb.y, -ca.y + cb.x);
  }
  __syncthreads();
  ring_dft_forward_f(buf, d, tw, twlog, bspec, u, T);
  if (va) {
    double* oa = map + int64_t(fa) * npix + g.start;
    double* ob = map + int64_t(fb) * npix + start_b;
    for (int j = u; j < N; j += T) {
      const float2 y = dft_get_f(buf, d, j);
      oa[j] = double(y.x);
      if (vb) ob[j] = double(y.y);
    }
  }
}

// adjoint: map [nf][npix] (float64) -> phase [R][mmax+1][nf] (complex64)
__global__ void ring_adjoint_f32(const RingInfo* __restrict__ rings, const int* __restrict__ ring_list, int R,
                                 const double* __restrict__ map, float2* __restrict__ phase, int mmax, int nf,
                                 int64_t npix, const float2* __restrict__ tw, int twlog,
                                 const float2* __restrict__ bs_spec, const int64_t* __restrict__ bs_off,
                               const float2* __restrict__ rot, const float2* __restrict__ chirp,
                               const int64_t* __restrict__ chirp_off, int T, int pack) {
  extern __shared__ float2 fbuf[];
  const int ir = ring_list[blockIdx.y];
  // partner of a packed FFT: the other component of the same map (pack), else the
  // same map on the mirror ring (same nphi and phi0; the list holds north rings)
  const int irb = pack ? ir : R - 1 - ir;
  const RingInfo g = rings[ir];
  const int64_t start_b = rings[irb].start;
  const RingDFTf d = make_dft(g, chirp, chirp_off);
  const float2* rotr = rot + int64_t(min(ir, R - 1 - ir)) * (mmax + 1);  // e^{i m phi0} of this ring
  const float2* bspec = d.bluestein ? bs_spec + bs_off[g.bs_slot] : nullptr;
  const int grp = threadIdx.x / T, u = threadIdx.x - grp * T;
  const int G = blockDim.x / T;
  const int unit = blockIdx.x * G + grp;
  const int fa = pack ? 2 * unit : unit, fb = pack ? fa + 1 : unit;
  const bool va = fa < nf, vb = pack ? fb < nf : (va && irb != ir);
  float2* buf = fbuf + size_t(grp) * d.M;
  const int N = d.N;
  {
    const double* ia = map + int64_t(va ? fa : 0) * npix + g.start;
    const double* ib = map + int64_t(vb ? fb : 0) * npix + (vb ? start_b : g.start);
    for (int j = u; j < N; j += T) buf[j] = make_float2(va ? float(ia[j]) : 0.f, vb ? float(ib[j]) : 0.f);
  }
  __syncthreads();
  ring_dft_forward_f(buf, d, tw, twlog, bspec, u, T);
  if (va) {
    float2* pha = phase + int64_t(ir) * (mmax + 1) * nf;
    float2* phb = phase + int64_t(irb) * (mmax + 1) * nf;
    for (int m = u; m <= mmax; m += T) {
      const int k = m % N, k2 = (N - k) % N;
      const float2 z = dft_get_f(buf, d, k), z2 = fconj2(dft_get_f(buf, d, k2));
      const float2 e = fconj2(rotr[m]);
      const float2 xa = make_float2(0.5f * (z.x + z2.x), 0.5f * (z.y + z2.y));
      // (z - z2) / (2i) = -i (z - z2) / 2
      const float2 xb = make_float2(0.5f * (z.y - z2.y), -0.5f * (z.x - z2.x));
      pha[int64_t(m) * nf + fa] = fmul2(xa, e);
      if (vb) phb[int64_t(m) * nf + fb] = fmul2(xb, e);
    }
  }
}

// synthesis -> pixel weights -> adjoint of the same rings, in place on the phases:
//   phase [R][mmax+1][nf] (complex64)  ->  P'_m = sum_j w_j map_j e^{-i m (phi0 + 2 pi j / nphi)}
// with map = the ring's synthesis of the phases and w the per-pixel weight of each field
// (weight [ncw][npix]: field a reads component 0, field b component 1 for a spin map, or
// component 0 on the mirror ring for spin 0).  The map never leaves shared memory: between the
// two DFTs each thread weights the pixels it owns (natural order for the second DFT: the
// bit-reversal of the first undone in place, in pairs).  The block reads every phase it writes
// before the first barrier, so in place is safe.
__global__ void ring_roundtrip_f32(const RingInfo* __restrict__ rings, const int* __restrict__ ring_list, int R,
                                   float2* __restrict__ phase, int mmax, int nf, const double* __restrict__ weight,
                                   int64_t npix, const float2* __restrict__ tw, int twlog,
                                   const float2* __restrict__ bs_spec, const int64_t* __restrict__ bs_off,
                                   const float2* __restrict__ rot, const float2* __restrict__ chirp,
                                   const int64_t* __restrict__ chirp_off, int T, int pack) {
  extern __shared__ float2 fbuf[];
  const int ir = ring_list[blockIdx.y];
  const int irb = pack ? ir : R - 1 - ir;
  const RingInfo g = rings[ir];
  const int64_t start_b = rings[irb].start;
  const RingDFTf d = make_dft(g, chirp, chirp_off);
  const float2* rotr = rot + int64_t(min(ir, R - 1 - ir)) * (mmax + 1);  // e^{i m phi0} of this ring
  const float2* bspec = d.bluestein ? bs_spec + bs_off[g.bs_slot] : nullptr;
  const int grp = threadIdx.x / T, u = threadIdx.x - grp * T;
  const int G = blockDim.x / T;
  const int unit = blockIdx.x * G + grp;
  const int fa = pack ? 2 * unit : unit, fb = pack ? fa + 1 : unit;
  const bool va = fa < nf, vb = pack ? fb < nf : (va && irb != ir);
  float2* buf = fbuf + size_t(grp) * d.M;
  const int N = d.N;
  float2* pha = phase + int64_t(ir) * (mmax + 1) * nf;
  float2* phb = phase + int64_t(irb) * (mmax + 1) * nf;
  for (int kk = u; kk < N; kk += T) {
    float2 ca = make_float2(0.f, 0.f), cb = ca;
    if (va) {
      for (int m = kk; m <= mmax; m += N) {
        const float2 e = rotr[m];
        ca = fadd2(ca, fmul2(pha[int64_t(m) * nf + fa], e));
        if (vb) cb = fadd2(cb, fmul2(phb[int64_t(m) * nf + fb], e));
      }
      for (int m = (kk == 0) ? N : N - kk; m <= mmax; m += N) {
        const float2 e = rotr[m];
        ca = fadd2(ca, fconj2(fmul2(pha[int64_t(m) * nf + fa], e)));
        if (vb) cb = fadd2(cb, fconj2(fmul2(phb[int64_t(m) * nf + fb], e)));
      }
    }
    if (kk == 0) { ca.y = 0.f; cb.y = 0.f; }
    buf[kk] = make_float2(ca.x + cb.y, -ca.y + cb.x);
  }
  __syncthreads();
  ring_dft_forward_f(buf, d, tw, twlog, bspec, u, T);
  // pixel j of field a is Re y_j, of field b Im y_j (y_j = dft_get_f(buf, d, j)); weight them
  const double* wa = weight + g.start;
  const double* wb = weight + (pack ? npix : 0) + start_b;
  if (!d.bluestein) {
    for (int j = u; j < N; j += T) {
      const int jr = bitrev_f(j, d.logM);
      if (j < jr) {
        const float2 yj = buf[jr], yr = buf[j];
        buf[j] = make_float2(va ? float(wa[j]) * yj.x : 0.f, vb ? float(wb[j]) * yj.y : 0.f);
        buf[jr] = make_float2(va ? float(wa[jr]) * yr.x : 0.f, vb ? float(wb[jr]) * yr.y : 0.f);
      } else if (j == jr) {
        const float2 yj = buf[j];
        buf[j] = make_float2(va ? float(wa[j]) * yj.x : 0.f, vb ? float(wb[j]) * yj.y : 0.f);
      }
    }
  } else {
    for (int j = u; j < N; j += T) {
      const float2 yj = dft_get_f(buf, d, j);
      buf[j] = make_float2(va ? float(wa[j]) * yj.x : 0.f, vb ? float(wb[j]) * yj.y : 0.f);
    }
  }
  __syncthreads();
  ring_dft_forward_f(buf, d, tw, twlog, bspec, u, T);
  if (va) {
    for (int m = u; m <= mmax; m += T) {
      const int k = m % N, k2 = (N - k) % N;
      const float2 z = dft_get_f(buf, d, k), z2 = fconj2(dft_get_f(buf, d, k2));
      const float2 e = fconj2(rotr[m]);
      const float2 xa = make_float2(0.5f * (z.x + z2.x), 0.5f * (z.y + z2.y));
      const float2 xb = make_float2(0.5f * (z.y - z2.y), -0.5f * (z.x - z2.x));
      pha[int64_t(m) * nf + fa] = fmul2(xa, e);
      if (vb) phb[int64_t(m) * nf + fb] = fmul2(xb, e);
    }
  }
}

static void fft_shape(int work_len, int nf, int pack, int& T, int& G, int& gy) {
  T = std::max(32, std::min(256, work_len / 4));
  G = std::max(1, 256 / T);
  const int units = pack ? (nf + 1) / 2 : nf;
  G = std::min(G, units);
  gy = (units + G - 1) / G;
}

int launch_ring_synth_f32(const Plan& P, const int* d_list, int nrings, int work_len, const float2* phase,
                          double* map, int nf, int pack, cudaStream_t st) {
  if (nrings == 0) return PS_OK;
  int T, G, gy;
  fft_shape(work_len, nf, pack, T, G, gy);
  if (nrings > 65535) return PS_ERR_INVALID;
  const size_t smem = size_t(work_len) * G * sizeof(float2);
  if (smem > 48 * 1024) {
    if (cudaFuncSetAttribute(ring_synth_f32, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
      return PS_ERR_CUDA;
  }
  int twlog = 0;
  while ((1 << twlog) < P.max_fft) ++twlog;
  StatScope sc(PS_K_FFT_SYNTH, 0.0, 0.0, st);
  ring_synth_f32<<<dim3(gy, nrings), T * G, smem, st>>>(P.d_rings, d_list, P.R, phase, map, P.mmax, nf, P.npix,
                                                         P.d_twiddle_f, twlog, P.d_bs_spec_f, P.d_bs_off,
                                                         P.d_rot_f, P.d_chirp_f, P.d_chirp_off, T, pack);
  PS_LAUNCH_CHECK();
  return PS_OK;
}

int launch_ring_adjoint_f32(const Plan& P, const int* d_list, int nrings, int work_len, const double* map,
                            float2* phase, int nf, int pack, cudaStream_t st) {
  if (nrings == 0) return PS_OK;
  int T, G, gy;
  fft_shape(work_len, nf, pack, T, G, gy);
  if (nrings > 65535) return PS_ERR_INVALID;
  const size_t smem = size_t(work_len) * G * sizeof(float2);
  if (smem > 48 * 1024) {
    if (cudaFuncSetAttribute(ring_adjoint_f32, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
      return PS_ERR_CUDA;
  }
  int twlog = 0;
  while ((1 << twlog) < P.max_fft) ++twlog;
  StatScope sc(PS_K_FFT_ADJOINT, 0.0, 0.0, st);
  ring_adjoint_f32<<<dim3(gy, nrings), T * G, smem, st>>>(P.d_rings, d_list, P.R, map, phase, P.mmax, nf, P.npix,
                                                           P.d_twiddle_f, twlog, P.d_bs_spec_f, P.d_bs_off,
                                                         P.d_rot_f, P.d_chirp_f, P.d_chirp_off, T, pack);
  PS_LAUNCH_CHECK();
  return PS_OK;
}

int launch_ring_roundtrip_f32(const Plan& P, const int* d_list, int nrings, int work_len, float2* phase,
                              const double* weight, int nf, int pack, cudaStream_t st) {
  if (nrings == 0) return PS_OK;
  int T, G, gy;
  fft_shape(work_len, nf, pack, T, G, gy);
  if (nrings > 65535) return PS_ERR_INVALID;
  const size_t smem = size_t(work_len) * G * sizeof(float2);
  if (smem > 48 * 1024) {
    if (cudaFuncSetAttribute(ring_roundtrip_f32, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
      return PS_ERR_CUDA;
  }
  int twlog = 0;
  while ((1 << twlog) < P.max_fft) ++twlog;
  // the pixel weights and the phases, read and written once
  const double bytes = double(P.npix) * 8.0 * (pack ? 2.0 : 1.0) + 2.0 * 8.0 * P.R * (P.mmax + 1) * nf;
  StatScope sc(PS_K_FFT_SYNTH, 0.0, bytes * double(nrings) / double(P.R), st);
  ring_roundtrip_f32<<<dim3(gy, nrings), T * G, smem, st>>>(P.d_rings, d_list, P.R, phase, P.mmax, nf, weight,
                                                             P.npix, P.d_twiddle_f, twlog, P.d_bs_spec_f, P.d_bs_off,
                                                             P.d_rot_f, P.d_chirp_f, P.d_chirp_off, T, pack);
  PS_LAUNCH_CHECK();
  return PS_OK;
}

}  // namespace ps
