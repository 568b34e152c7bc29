// Shared definitions of the libpscuda kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cmath>

#include "../../include/pscuda.h"

namespace ps {

// ---------------------------------------------------------------------------
// HEALPix ring, as the kernels see it.  The longitude of the first pixel is
// phi0 = pi * phi_num / phi_den (phi_num in {0, 1}), kept as a rational so that
// e^{i m phi0} is evaluated with an exact integer argument reduction.
struct RingInfo {
  double z;        // cos(theta)
  double omz;      // 1 - z (accurate near the north pole)
  double opz;      // 1 + z (accurate near the south pole)
  double sth;      // sin(theta)
  int64_t start;   // first pixel of the ring
  int nphi;        // pixels in the ring
  int phi_num;     // phi0 = pi * phi_num / phi_den
  int phi_den;
  int bs_slot;     // index of the Bluestein kernel spectrum (-1: power-of-two length)
  int bs_m;        // Bluestein FFT length (power of two), 0 for power-of-two rings
  int pad;
};

// Bluestein chirp spectra, one per distinct non-power-of-two ring length.
struct BluesteinTable {
  const double2* spec;     // concatenated FFT_M(b) arrays
  const int64_t* offset;   // offset of slot s in spec
};

// Legendre seed normalisation for spin s at order m, as mantissa * 2^exp.
struct SeedNorm { double v; int e; int pad; };

struct Plan {
  int nside, lmax, mmax, R, Rh, prec, spin_mask;
  int64_t npix, nalm;
  int max_fft;              // largest FFT length used (power of two)
  RingInfo* d_rings;        // [R]
  double* d_mnorm0;         // [mmax+1] spin-0 seed normalisation
  SeedNorm* d_seed[4];      // [mmax+1] per spin 1..3 (index 1..3), null if not in spin_mask
  double2* d_twiddle;       // [max_fft/2] e^{-2 pi i k / max_fft}
  double2* d_bs_spec;       // Bluestein spectra (FP64)
  float2* d_twiddle_f;      // FP32 copies for the mixed-precision ring transforms
  float2* d_bs_spec_f;
  // mixed plans: e^{i m phi0} of every north ring (the mirror ring has the same phi0),
  // [Rh][mmax+1], and the Bluestein chirps e^{-i pi j^2 / N}, j < N, of every slot
  float2* d_rot_f;
  float2* d_chirp_f;
  int64_t* d_chirp_off;
  int* d_err;               // device error flag raised by kernels whose bounded waits expired
  int64_t* d_bs_off;        // [nslots]
  int n_bs_slots;
  int64_t bs_total;
  int num_sms;
  // maps per CTA of the Legendre stages, [direction 0 synthesis / 1 adjoint][spin];
  // 0 = the launcher's own choice (set by ps_plan_set_tile, e.g. from the autotuner)
  int tile[2][4];
  // Legendre tables of a mixed-precision plan (ps_plan_build_table), per spin; null when
  // not built.  d_tab_off [mmax+2]: first table block of each order; d_tab_work: the
  // (m, first block) list of the table adjoint's CTAs.
  float* d_tab[4];
  int64_t* d_tab_off;
  int2* d_tab_work;
  int tab_nwork;
  // format of each built table (PS_TAB_TF32X3 or PS_TAB_BF16X3) and of the tables built next
  int tab_fmt[4];
  int tab_fmt_build;
};

// ---------------------------------------------------------------------------
// complex helpers (double2 = re, im)
__host__ __device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__host__ __device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ double2 cfma(double s, double2 a, double2 acc) {
  return make_double2(fma(s, a.x, acc.x), fma(s, a.y, acc.y));
}

__host__ __device__ __forceinline__ int64_t alm_index(int l, int m, int lmax) {
  return int64_t(m) * (2 * lmax + 1 - m) / 2 + l;
}

// Large-exponent bookkeeping of the Legendre recurrences: true value is
// v * 2^(SCALE_BITS * k) with k <= 0; while k < 0 the value is below
// 2^-(SCALE_BITS/2) and contributes nothing at FP64 precision.
constexpr int SCALE_BITS = 800;
#define PS_FTHRESH 0x1p400
#define PS_FSMALL 0x1p-800

// value = v * 2^e with v in [0.5, 1)
struct Scaled { double v; int e; };

__host__ __device__ __forceinline__ Scaled snorm(double x) {
  int e; double v = frexp(x, &e); Scaled r; r.v = v; r.e = e; return r;
}
__host__ __device__ __forceinline__ Scaled smul(Scaled a, Scaled b) {
  Scaled r = snorm(a.v * b.v); r.e += a.e + b.e; return r;
}
__host__ __device__ __forceinline__ Scaled spow(double x, int n) {  // x > 0, n >= 0
  Scaled r; r.v = 0.5; r.e = 1;
  Scaled b = snorm(x);
  while (n) { if (n & 1) r = smul(r, b); b = smul(b, b); n >>= 1; }
  return r;
}
// Split a Scaled into (v, k): value = v * 2^(SCALE_BITS k), k <= 0, and for
// k < 0 |v| <= 2^(SCALE_BITS/2).
__host__ __device__ __forceinline__ void to_kscale(Scaled s, double& v, int& k) {
  if (s.v == 0.0) { v = 0.0; k = 0; return; }
  int e = s.e;
  k = 0;
  if (e <= -SCALE_BITS / 2) {
    int steps = (-SCALE_BITS / 2 - e) / SCALE_BITS + 1;
    e += steps * SCALE_BITS;
    k = -steps;
  }
  v = ldexp(s.v, e);
}

// Streaming-multiprocessor count of the current device (read once per device and
// kept), for grid caps that a workspace query and its launch must agree on.
inline int device_sms() {
  static int cached[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (!cached[dev]) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) return 148;
    cached[dev] = n;
  }
  return cached[dev];
}

}  // namespace ps

// launch-error helper for the C-ABI layer
#define PS_LAUNCH_CHECK()                                          \
  do {                                                             \
    cudaError_t _e = cudaGetLastError();                           \
    if (_e != cudaSuccess) return PS_ERR_CUDA;                     \
  } while (0)
