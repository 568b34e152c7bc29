// Plans and the SHT entry points of the C ABI (include/pscuda.h).
//
// A plan holds the read-only tables of one (nside, lmax) geometry: the
// HEALPix RING table, the Legendre seed normalisations, the FFT twiddles,
// the Bluestein chirp spectra and the grouping of rings into FFT length
// classes.  Everything else (transposed alm, the ring/order "phase" array,
// the adjoint's per-tile partial sums) lives in caller-owned workspace.
#include <vector>
#include <complex>
#include <map>
#include <algorithm>
#include <new>

#include "ps_common.cuh"

namespace ps {
int launch_legendre_synth_f64(const Plan& P, const double2* almT, double2* phase, int B, int spin, cudaStream_t st);
int launch_legendre_adjoint_f64(const Plan& P, const double2* phase, double2* partial, int B, int bofs, int Bc,
                                int spin, cudaStream_t st);
int adjoint_tiles(const Plan& P);
int launch_alm_to_T(const double2* alm, double2* almT, int B, int ncomp, int64_t nalm, int sms, cudaStream_t st);
int launch_reduce_partials(const double2* partial, double2* alm, int ntiles, int B, int ncomp, int64_t nalm,
                           double scale, int bofs, int sms, cudaStream_t st);
int launch_ring_synth_f64(const Plan& P, const int* d_list, int nrings, int work_len, const double2* phase,
                          double* map, int nf, int pack, cudaStream_t st);
int launch_ring_adjoint_f64(const Plan& P, const int* d_list, int nrings, int work_len, const double* map,
                            double2* phase, int nf, int pack, cudaStream_t st);
int launch_ring_synth_f32(const Plan& P, const int* d_list, int nrings, int work_len, const float2* phase,
                          double* map, int nf, int pack, cudaStream_t st);
int launch_ring_adjoint_f32(const Plan& P, const int* d_list, int nrings, int work_len, const double* map,
                            float2* phase, int nf, int pack, cudaStream_t st);
int launch_legendre_synth_tc(const Plan& P, const double2* almT, float2* phase, int B, int spin, int* err_flag,
                             cudaStream_t st);
int launch_legendre_adjoint_mx(const Plan& P, const float2* phase, float2* partial, int B, int bofs, int Bc,
                               int spin, cudaStream_t st);
int mx_adjoint_tiles(const Plan& P);
int launch_reduce_partials_f32(const float2* partial, double2* alm, int ntiles, int B, int ncomp, int64_t nalm,
                               double scale, int bofs, int sms, cudaStream_t st);
size_t tab_bytes(int Rh, int lmax, int mmax, int spin);
size_t tab3_bytes(int Rh, int lmax, int mmax, int spin);
int launch_tab3_gen(const Plan& P, int spin, const int64_t* d_blockoff, uint16_t* table, cudaStream_t st);
void tab_blockoff(int lmax, int mmax, std::vector<int64_t>& off);
void tab_adj_work(int lmax, int mmax, std::vector<int2>& work);
int launch_tab_gen(const Plan& P, int spin, const int64_t* d_blockoff, float* table, cudaStream_t st);
int launch_tab_synth(const Plan& P, const float* table, const int64_t* d_blockoff, int Rh_table, int toff,
                     const double2* almT, float2* phase, int B, int spin, int* err_flag, cudaStream_t st, int fmt);
int launch_tab_adj(const Plan& P, const float* table, const int64_t* d_blockoff, const int2* d_work, int nwork,
                   int Rh_table, int toff, const float2* phase, double2* alm, int B, int spin, double scale,
                   int64_t out_stride, const double* lscale, int* err_flag, cudaStream_t st, int fmt);
}  // namespace ps

struct ps_plan {
  ps::Plan p;
  // a ring-band plan (ps_plan_band) shares its parent's tables and runs the
  // Legendre stages only; it reads the parent's Legendre tables (built before or
  // after the band plan) through `parent`
  bool is_band = false;
  const ps_plan* parent = nullptr;
  // Legendre tables owned by this plan (ps_plan_build_table), per spin
  void* tab_alloc[4] = {nullptr, nullptr, nullptr, nullptr};
  void* tab_meta = nullptr;  // d_tab_off and d_tab_work in one allocation
  // FFT length classes: rings with the same work length share a launch
  std::vector<int> cls_len, cls_off, cls_cnt;
  std::vector<int> cls_off_n, cls_cnt_n;  // the north rings (and the equator ring) of each class
  int* d_ring_lists = nullptr;
  std::vector<void*> owned;  // device allocations to free
};

namespace {

bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }
int next_pow2(int n) { int m = 1; while (m < n) m <<= 1; return m; }

// host radix-2 FFT (sign -1), natural order in and out; used once per plan to
// build the Bluestein kernel spectra
void host_fft(std::vector<std::complex<double>>& a) {
  const int n = (int)a.size();
  for (int i = 1, j = 0; i < n; ++i) {
    int bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) std::swap(a[i], a[j]);
  }
  for (int len = 2; len <= n; len <<= 1) {
    for (int j = 0; j < len / 2; ++j) {
      const double ang = -2.0 * M_PI * double(j) / double(len);
      const std::complex<double> w(std::cos(ang), std::sin(ang));
      for (int i = 0; i < n; i += len) {
        const std::complex<double> u = a[i + j], v = a[i + j + len / 2] * w;
        a[i + j] = u + v;
        a[i + j + len / 2] = u - v;
      }
    }
  }
}

int host_bitrev(int i, int logn) {
  int r = 0;
  for (int b = 0; b < logn; ++b) { r = (r << 1) | (i & 1); i >>= 1; }
  return r;
}

template <class T>
T* dev_upload(ps_plan* pl, const std::vector<T>& v, int& err) {
  if (v.empty()) return nullptr;
  void* d = nullptr;
  if (cudaMalloc(&d, v.size() * sizeof(T)) != cudaSuccess) { err = PS_ERR_NOMEM; return nullptr; }
  pl->owned.push_back(d);
  if (cudaMemcpy(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess) err = PS_ERR_CUDA;
  return static_cast<T*>(d);
}

// sqrt of a Scaled value
ps::Scaled ssqrt(ps::Scaled s) {
  double v = s.v; int e = s.e;
  if (e & 1) { v *= 2.0; e -= 1; }
  ps::Scaled r = ps::snorm(std::sqrt(v));
  r.e += e / 2;
  return r;
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// The Legendre table a mixed-precision plan's transforms of `spin` read, if any: the
// plan's own, or for a band plan its parent's at the band's ring offset.
struct TabRef {
  const float* tab;
  const int64_t* off;
  const int2* work;
  int nwork, Rh_table, toff, fmt;
};
bool table_for(const ps_plan* plan, int spin, TabRef& t) {
  const ps_plan* owner = plan->is_band ? plan->parent : plan;
  if (!owner || plan->p.prec != PS_PREC_MIXED || !owner->p.d_tab[spin]) return false;
  t.tab = owner->p.d_tab[spin];
  t.off = owner->p.d_tab_off;
  t.work = owner->p.d_tab_work;
  t.nwork = owner->p.tab_nwork;
  t.Rh_table = owner->p.Rh;
  t.toff = owner->p.Rh - plan->p.Rh;
  t.fmt = owner->p.tab_fmt[spin];
  return true;
}

}  // namespace

extern "C" {

const char* ps_error_string(int code) {
  switch (code) {
    case PS_OK: return "ok";
    case PS_ERR_INVALID: return "invalid argument";
    case PS_ERR_UNSUPPORTED: return "unsupported configuration";
    case PS_ERR_NOMEM: return "device allocation failed";
    case PS_ERR_CUDA: return "CUDA runtime error";
    case PS_ERR_WORKSPACE: return "workspace too small";
    case PS_ERR_NOT_CONVERGED: return "solver did not converge";
    default: return "unknown error";
  }
}

int ps_version(void) { return 100; }

int ps_device_sm_count(int* count) {
  if (!count) return PS_ERR_INVALID;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return PS_ERR_CUDA;
  if (cudaDeviceGetAttribute(count, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return PS_ERR_CUDA;
  return PS_OK;
}

int ps_plan_create(int nside, int lmax, int mmax, int spin_mask, int prec, ps_plan** out) {
  if (!out) return PS_ERR_INVALID;
  *out = nullptr;
  if (nside < 1 || nside > 8192 || lmax < 0 || mmax != lmax || (prec != PS_PREC_FP64 && prec != PS_PREC_MIXED))
    return PS_ERR_INVALID;
  if (spin_mask & ~0xF) return PS_ERR_UNSUPPORTED;  // spins 0..3
  ps_plan* pl = new (std::nothrow) ps_plan();
  if (!pl) return PS_ERR_NOMEM;
  ps::Plan& P = pl->p;
  P.nside = nside; P.lmax = lmax; P.mmax = mmax; P.prec = prec; P.spin_mask = spin_mask | 1;
  P.R = 4 * nside - 1; P.Rh = 2 * nside;
  P.npix = 12 * int64_t(nside) * nside;
  P.nalm = int64_t(lmax + 1) * (lmax + 2) / 2;
  for (int s = 0; s < 4; ++s) { P.d_seed[s] = nullptr; P.d_tab[s] = nullptr; P.tab_fmt[s] = PS_TAB_TF32X3; }
  P.tab_fmt_build = PS_TAB_TF32X3;
  P.d_tab_off = nullptr;
  P.d_tab_work = nullptr;
  P.tab_nwork = 0;
  for (int d = 0; d < 2; ++d)
    for (int s = 0; s < 4; ++s) P.tile[d][s] = 0;
  if (ps_device_sm_count(&P.num_sms) != PS_OK) { delete pl; return PS_ERR_CUDA; }
  int err = PS_OK;

  // ---- ring table (HEALPix RING, Gorski et al. 2005)
  std::vector<ps::RingInfo> rings(P.R);
  std::map<int, int> bs_slot;  // nphi -> slot
  std::vector<int> bs_n;
  const int64_t ns = nside;
  for (int ir = 0; ir < P.R; ++ir) {
    const int64_t i = ir + 1;
    const bool north = i <= 2 * ns;
    const int64_t ii = north ? i : 4 * ns - i;
    ps::RingInfo g{};
    if (ii < ns) {
      const double t = double(ii * ii) / (3.0 * double(ns * ns));
      g.z = north ? 1.0 - t : t - 1.0;
      g.omz = north ? t : 2.0 - t;
      g.opz = north ? 2.0 - t : t;
      g.sth = std::sqrt(t * (2.0 - t));
      g.nphi = int(4 * ii);
      g.phi_num = 1; g.phi_den = int(4 * ii);
      g.start = north ? 2 * ii * (ii - 1) : P.npix - 2 * ii * (ii + 1);
    } else {
      const double z = double(2 * ns - i) * 2.0 / (3.0 * double(ns));
      g.z = z; g.omz = 1.0 - z; g.opz = 1.0 + z;
      g.sth = std::sqrt(g.omz * g.opz);
      g.nphi = int(4 * ns);
      g.phi_num = ((i - ns) % 2 == 0) ? 1 : 0;
      g.phi_den = int(4 * ns);
      g.start = 2 * ns * (ns - 1) + (i - ns) * 4 * ns;
    }
    if (is_pow2(g.nphi)) { g.bs_slot = -1; g.bs_m = 0; }
    else {
      auto it = bs_slot.find(g.nphi);
      if (it == bs_slot.end()) { it = bs_slot.emplace(g.nphi, (int)bs_n.size()).first; bs_n.push_back(g.nphi); }
      g.bs_slot = it->second;
      g.bs_m = next_pow2(2 * g.nphi - 1);
    }
    rings[ir] = g;
  }

  // ---- FFT classes and twiddles
  std::map<int, std::vector<int>> classes;
  int max_fft = 2;
  for (int ir = 0; ir < P.R; ++ir) {
    const int w = rings[ir].bs_slot >= 0 ? rings[ir].bs_m : rings[ir].nphi;
    classes[w].push_back(ir);
    max_fft = std::max(max_fft, w);
  }
  P.max_fft = max_fft;
  {
    // the FP64 ring transforms keep a ring's work array (max_fft complex values) in shared memory;
    // the mixed-precision path uses FP32 work arrays (half the size)
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const size_t elem = (prec == PS_PREC_FP64) ? sizeof(double2) : sizeof(float2);
    if (size_t(max_fft) * elem > size_t(optin)) { delete pl; return PS_ERR_UNSUPPORTED; }
  }
  std::vector<int> lists;
  for (auto& kv : classes) {
    pl->cls_len.push_back(kv.first);
    pl->cls_off.push_back((int)lists.size());
    pl->cls_cnt.push_back((int)kv.second.size());
    // largest rings first inside a class does not matter: all have equal work
    lists.insert(lists.end(), kv.second.begin(), kv.second.end());
  }
  for (auto& kv : classes) {
    pl->cls_off_n.push_back((int)lists.size());
    int n = 0;
    for (int ir : kv.second)
      if (ir <= P.R - 1 - ir) { lists.push_back(ir); ++n; }
    pl->cls_cnt_n.push_back(n);
  }
  std::vector<double2> tw(max_fft / 2);
  for (int k = 0; k < max_fft / 2; ++k) {
    const double ang = -2.0 * M_PI * double(k) / double(max_fft);
    tw[k] = make_double2(std::cos(ang), std::sin(ang));
  }
  // ---- Bluestein spectra: b_n = e^{+i pi n^2 / N}, |n| < N, wrapped to M; FFT_M, bit-reversed order
  std::vector<double2> bs_spec;
  std::vector<int64_t> bs_off;
  for (int N : bs_n) {
    const int M = next_pow2(2 * N - 1);
    int logM = 0; while ((1 << logM) < M) ++logM;
    std::vector<std::complex<double>> b(M, 0.0);
    for (int n = 0; n < N; ++n) {
      const int64_t q = (int64_t(n) * n) % (2 * int64_t(N));
      const double ang = M_PI * double(q) / double(N);
      const std::complex<double> v(std::cos(ang), std::sin(ang));
      b[n] = v;
      if (n > 0) b[M - n] = v;
    }
    host_fft(b);
    bs_off.push_back((int64_t)bs_spec.size());
    const size_t o = bs_spec.size();
    bs_spec.resize(o + M);
    for (int p = 0; p < M; ++p) {
      const std::complex<double> v = b[host_bitrev(p, logM)];
      bs_spec[o + p] = make_double2(v.real(), v.imag());
    }
  }
  P.n_bs_slots = (int)bs_n.size();
  P.bs_total = (int64_t)bs_spec.size();

  // ---- Legendre seed normalisations
  std::vector<double> mnorm(mmax + 1);
  {
    double p = 1.0;
    for (int m = 0; m <= mmax; ++m) {
      if (m > 0) p *= (2.0 * m - 1.0) / (2.0 * m);
      mnorm[m] = std::sqrt((2.0 * m + 1.0) / (4.0 * M_PI) * p);
    }
  }
  std::vector<ps::SeedNorm> seeds[4];
  for (int s = 1; s <= 3; ++s) {
    if (!((spin_mask >> s) & 1)) continue;
    seeds[s].resize(mmax + 1);
    // C(2m, m+s) for m >= s, incrementally; C(2s, s+m) for m < s directly
    ps::Scaled binom = ps::snorm(1.0);
    for (int m = 0; m <= mmax; ++m) {
      ps::Scaled nrm;
      if (m < s) {
        ps::Scaled c = ps::snorm(1.0);
        for (int j = 1; j <= s - m; ++j) c = ps::smul(c, ps::snorm(double(s + m + j) / double(j)));
        nrm = ps::smul(c, ps::snorm((2.0 * s + 1.0) / (4.0 * M_PI)));
      } else {
        if (m > s)
          binom = ps::smul(binom, ps::snorm((2.0 * m) * (2.0 * m - 1.0) / (double(m + s) * double(m - s))));
        nrm = ps::smul(binom, ps::snorm((2.0 * m + 1.0) / (4.0 * M_PI)));
      }
      ps::Scaled r = ssqrt(nrm);
      seeds[s][m].v = r.v; seeds[s][m].e = r.e; seeds[s][m].pad = 0;
    }
  }

  P.d_rings = dev_upload(pl, rings, err);
  P.d_mnorm0 = dev_upload(pl, mnorm, err);
  for (int s = 1; s <= 3; ++s) if (!seeds[s].empty()) P.d_seed[s] = dev_upload(pl, seeds[s], err);
  P.d_twiddle = dev_upload(pl, tw, err);
  P.d_bs_spec = dev_upload(pl, bs_spec, err);
  {
    std::vector<float2> twf(tw.size()), bsf(bs_spec.size());
    for (size_t i = 0; i < tw.size(); ++i) twf[i] = make_float2(float(tw[i].x), float(tw[i].y));
    for (size_t i = 0; i < bs_spec.size(); ++i) bsf[i] = make_float2(float(bs_spec[i].x), float(bs_spec[i].y));
    P.d_twiddle_f = dev_upload(pl, twf, err);
    P.d_bs_spec_f = dev_upload(pl, bsf, err);
    std::vector<int> zero(1, 0);
    P.d_err = dev_upload(pl, zero, err);
  }
  P.d_bs_off = dev_upload(pl, bs_off, err);
  P.d_rot_f = nullptr;
  P.d_chirp_f = nullptr;
  P.d_chirp_off = nullptr;
  if (prec == PS_PREC_MIXED) {
    // ring rotations and Bluestein chirps of the FP32 ring transforms, from exact integer
    // argument reduction in FP64 (so the kernels evaluate no sincos)
    std::vector<float2> rot(size_t(P.Rh) * (mmax + 1));
    for (int rp = 0; rp < P.Rh; ++rp) {
      const int64_t num = rings[rp].phi_num, den = rings[rp].phi_den;
      for (int m = 0; m <= mmax; ++m) {
        const int64_t q = (int64_t(m) * num) % (2 * den);
        const double a = M_PI * double(q) / double(den);
        rot[size_t(rp) * (mmax + 1) + m] = make_float2(float(std::cos(a)), float(std::sin(a)));
      }
    }
    std::vector<float2> chirp;
    std::vector<int64_t> chirp_off;
    for (int N : bs_n) {
      chirp_off.push_back((int64_t)chirp.size());
      for (int j = 0; j < N; ++j) {
        const int64_t q = (int64_t(j) * j) % (2 * int64_t(N));
        const double a = -M_PI * double(q) / double(N);
        chirp.push_back(make_float2(float(std::cos(a)), float(std::sin(a))));
      }
    }
    P.d_rot_f = dev_upload(pl, rot, err);
    P.d_chirp_f = dev_upload(pl, chirp, err);
    P.d_chirp_off = dev_upload(pl, chirp_off, err);
  }
  pl->d_ring_lists = dev_upload(pl, lists, err);
  if (err != PS_OK) { ps_plan_destroy(pl); return err; }
  *out = pl;
  return PS_OK;
}

// Allowed maps-per-CTA of the Legendre stages: {prec}{direction}{spin 0, spin s}
static bool tile_allowed(int prec, int direction, int spin, int tile) {
  if (tile == 0) return true;
  const bool s0 = spin == 0;
  if (prec == PS_PREC_MIXED) {
    if (direction == 0) return s0 ? (tile == 8 || tile == 16 || tile == 32) : (tile == 4 || tile == 8);
    return s0 ? (tile == 1 || tile == 8) : (tile == 1 || tile == 4);
  }
  if (direction == 0) return s0 ? (tile == 1 || tile == 4) : (tile == 1 || tile == 2);
  return s0 ? (tile == 1 || tile == 4) : tile == 1;
}

int ps_plan_set_tile(ps_plan* plan, int direction, int spin, int tile) {
  if (!plan || direction < 0 || direction > 1 || spin < 0 || spin > 3) return PS_ERR_INVALID;
  if (!tile_allowed(plan->p.prec, direction, spin, tile)) return PS_ERR_UNSUPPORTED;
  plan->p.tile[direction][spin] = tile;
  return PS_OK;
}

int ps_plan_band(const ps_plan* full, int nrings_north, ps_plan** out) {
  if (!full || !out || full->is_band) return PS_ERR_INVALID;
  const ps::Plan& F = full->p;
  if (nrings_north < 1 || nrings_north > F.Rh || (F.R & 1) == 0) return PS_ERR_INVALID;
  ps_plan* pl = new ps_plan();
  pl->p = F;
  pl->is_band = true;
  pl->parent = full;
  for (int d = 0; d < 2; ++d)
    for (int s = 0; s < 4; ++s) pl->p.tile[d][s] = 0;  // the launchers' own choice on the band
  // north rings [Rh - k, Rh) (the last one is the equator ring) and their mirrors
  pl->p.d_rings = F.d_rings + (F.Rh - nrings_north);
  pl->p.Rh = nrings_north;
  pl->p.R = 2 * nrings_north - 1;
  *out = pl;
  return PS_OK;
}

static size_t leg_ws_bytes(const ps_plan* plan, int batch, int spin, int adjoint);

int ps_legendre_workspace_bytes(const ps_plan* plan, int batch, int spin, int adjoint, size_t* bytes) {
  if (!plan || !bytes || batch < 0 || spin < 0 || spin > 3) return PS_ERR_INVALID;
  *bytes = leg_ws_bytes(plan, batch, spin, adjoint);
  return PS_OK;
}

int ps_plan_destroy(ps_plan* plan) {
  if (!plan) return PS_ERR_INVALID;
  if (!plan->is_band) {
    for (void* d : plan->owned) cudaFree(d);
    for (void* d : plan->tab_alloc) if (d) cudaFree(d);
    if (plan->tab_meta) cudaFree(plan->tab_meta);
  }
  delete plan;
  return PS_OK;
}

int ps_plan_table_bytes(const ps_plan* plan, int spin, size_t* bytes) {
  if (!plan || !bytes || spin < 0 || spin > 3) return PS_ERR_INVALID;
  const ps::Plan& P = plan->p;
  *bytes = P.tab_fmt_build == PS_TAB_BF16X3 ? ps::tab3_bytes(P.Rh, P.lmax, P.mmax, spin)
                                             : ps::tab_bytes(P.Rh, P.lmax, P.mmax, spin);
  return PS_OK;
}

int ps_plan_set_table_format(ps_plan* plan, int format) {
  if (!plan || (format != PS_TAB_TF32X3 && format != PS_TAB_BF16X3)) return PS_ERR_INVALID;
  if (plan->is_band || plan->p.prec != PS_PREC_MIXED) return PS_ERR_UNSUPPORTED;
  plan->p.tab_fmt_build = format;
  return PS_OK;
}

int ps_plan_has_table(const ps_plan* plan, int spin, int* has) {
  if (!plan || !has || spin < 0 || spin > 3) return PS_ERR_INVALID;
  const ps_plan* owner = plan->is_band ? plan->parent : plan;
  *has = owner && owner->p.d_tab[spin] != nullptr;
  return PS_OK;
}

int ps_plan_build_table(ps_plan* plan, int spin, cudaStream_t stream) {
  if (!plan || spin < 0 || spin > 3) return PS_ERR_INVALID;
  if (plan->is_band || plan->p.prec != PS_PREC_MIXED) return PS_ERR_UNSUPPORTED;
  ps::Plan& P = plan->p;
  if (spin > 0 && !P.d_seed[spin]) return PS_ERR_INVALID;
  if (P.d_tab[spin]) return PS_OK;
  if (!plan->tab_meta) {
    std::vector<int64_t> off;
    std::vector<int2> work;
    ps::tab_blockoff(P.lmax, P.mmax, off);
    ps::tab_adj_work(P.lmax, P.mmax, work);
    const size_t off_bytes = align256(off.size() * sizeof(int64_t));
    void* d = nullptr;
    if (cudaMalloc(&d, off_bytes + work.size() * sizeof(int2)) != cudaSuccess) {
      cudaGetLastError();
      return PS_ERR_NOMEM;
    }
    if (cudaMemcpy(d, off.data(), off.size() * sizeof(int64_t), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(static_cast<char*>(d) + off_bytes, work.data(), work.size() * sizeof(int2),
                   cudaMemcpyHostToDevice) != cudaSuccess) {
      cudaFree(d);
      return PS_ERR_CUDA;
    }
    plan->tab_meta = d;
    P.d_tab_off = static_cast<int64_t*>(d);
    P.d_tab_work = reinterpret_cast<int2*>(static_cast<char*>(d) + off_bytes);
    P.tab_nwork = int(work.size());
  }
  void* t = nullptr;
  const int fmt = P.tab_fmt_build;
  const size_t tb = fmt == PS_TAB_BF16X3 ? ps::tab3_bytes(P.Rh, P.lmax, P.mmax, spin)
                                         : ps::tab_bytes(P.Rh, P.lmax, P.mmax, spin);
  if (cudaMalloc(&t, tb) != cudaSuccess) {
    cudaGetLastError();
    return PS_ERR_NOMEM;
  }
  const int rc = fmt == PS_TAB_BF16X3 ? ps::launch_tab3_gen(P, spin, P.d_tab_off, static_cast<uint16_t*>(t), stream)
                                      : ps::launch_tab_gen(P, spin, P.d_tab_off, static_cast<float*>(t), stream);
  if (rc != PS_OK) { cudaFree(t); return rc; }
  P.tab_fmt[spin] = fmt;
  plan->tab_alloc[spin] = t;
  P.d_tab[spin] = static_cast<float*>(t);
  return PS_OK;
}

int ps_plan_drop_tables(ps_plan* plan) {
  if (!plan) return PS_ERR_INVALID;
  if (plan->is_band) return PS_ERR_UNSUPPORTED;
  if (cudaDeviceSynchronize() != cudaSuccess) return PS_ERR_CUDA;
  for (int s = 0; s < 4; ++s) {
    if (plan->tab_alloc[s]) cudaFree(plan->tab_alloc[s]);
    plan->tab_alloc[s] = nullptr;
    plan->p.d_tab[s] = nullptr;
  }
  return PS_OK;
}

int ps_plan_error_flag(const ps_plan* plan, int* value, int reset) {
  if (!plan || !value) return PS_ERR_INVALID;
  if (cudaMemcpy(value, plan->p.d_err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return PS_ERR_CUDA;
  if (reset && cudaMemset(plan->p.d_err, 0, sizeof(int)) != cudaSuccess) return PS_ERR_CUDA;
  return PS_OK;
}

int ps_plan_info(const ps_plan* plan, int* nside, int* lmax, int64_t* npix, int64_t* nalm) {
  if (!plan) return PS_ERR_INVALID;
  if (nside) *nside = plan->p.nside;
  if (lmax) *lmax = plan->p.lmax;
  if (npix) *npix = plan->p.npix;
  if (nalm) *nalm = plan->p.nalm;
  return PS_OK;
}

// maps per Legendre-adjoint pass: the per-ring-tile partial sums of one pass
// bound the adjoint's workspace independently of the batch size (at most about
// 4 GiB of partials per pass, at least one map)
static int adjoint_chunk(const ps::Plan& P, int batch, int spin) {
  int c = (P.prec == PS_PREC_MIXED) ? (spin == 0 ? 16 : 8) : (spin == 0 ? 8 : 4);
  const int tiles = (P.prec == PS_PREC_MIXED) ? ps::mx_adjoint_tiles(P) : ps::adjoint_tiles(P);
  const double per_map = double(tiles) * double(P.nalm) * (spin == 0 ? 1 : 2) *
                         (P.prec == PS_PREC_MIXED ? sizeof(float2) : sizeof(double2));
  const int cap = int(4294967296.0 / per_map);
  if (c > cap) c = cap < 1 ? 1 : cap;
  return batch < c ? batch : c;
}

static size_t sht_ws_bytes(const ps_plan* plan, int batch, int spin, int adjoint) {
  const ps::Plan& P = plan->p;
  const size_t ncomp = spin == 0 ? 1 : 2;
  const size_t nf = size_t(batch) * ncomp;
  const size_t phase = align256(size_t(P.R) * (P.mmax + 1) * nf * sizeof(double2));
  if (!adjoint) return align256(size_t(P.nalm) * nf * sizeof(double2)) + phase;
  TabRef tr;
  if (table_for(plan, spin, tr)) return phase;  // the table adjoint writes alm directly
  const size_t nfc = size_t(adjoint_chunk(P, batch, spin)) * ncomp;
  return phase + align256(size_t(ps::adjoint_tiles(P)) * P.nalm * nfc * sizeof(double2));
}

// Legendre stages alone (phase in and out in the caller's memory, complex128).
// A mixed-precision plan runs its tensor-core synthesis / FP32 adjoint kernels
// with the phases converted to complex64 in the workspace.
static int fp64_adjoint_chunk(int batch, int spin) {
  const int c = spin == 0 ? 8 : 4;
  return batch < c ? batch : c;
}

namespace {
__global__ void phase_f32_to_f64(const float2* __restrict__ in, double2* __restrict__ out, int64_t n) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const float2 v = in[i];
    out[i] = make_double2(double(v.x), double(v.y));
  }
}
__global__ void phase_f64_to_f32(const double2* __restrict__ in, float2* __restrict__ out, int64_t n) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const double2 v = in[i];
    out[i] = make_float2(float(v.x), float(v.y));
  }
}
int convert_grid(int64_t n, int sms) {
  const int64_t need = (n + 255) / 256, cap = int64_t(sms) * 8;
  return int(need < cap ? need : cap);
}
}  // namespace

static size_t leg_ws_bytes(const ps_plan* plan, int batch, int spin, int adjoint) {
  const ps::Plan& P = plan->p;
  const size_t ncomp = spin == 0 ? 1 : 2;
  const size_t nf = size_t(batch) * ncomp;
  const bool mixed = P.prec == PS_PREC_MIXED;
  const size_t phase32 = mixed ? align256(size_t(P.R) * (P.mmax + 1) * nf * sizeof(float2)) : 0;
  if (!adjoint) return align256(size_t(P.nalm) * nf * sizeof(double2)) + phase32;
  TabRef tr;
  if (table_for(plan, spin, tr)) return phase32;
  if (mixed) {
    const size_t nfc = size_t(adjoint_chunk(P, batch, spin)) * ncomp;
    return phase32 + align256(size_t(ps::mx_adjoint_tiles(P)) * P.nalm * nfc * sizeof(float2));
  }
  const size_t nfc = size_t(fp64_adjoint_chunk(batch, spin)) * ncomp;
  return align256(size_t(ps::adjoint_tiles(P)) * P.nalm * nfc * sizeof(double2));
}

int ps_legendre_synthesis(const ps_plan* plan, const double* alm, double* phase, int batch, int spin,
                          void* workspace, size_t workspace_bytes, cudaStream_t stream) {
  if (!plan || batch < 0 || spin < 0 || spin > 3) return PS_ERR_INVALID;
  if (batch == 0) return PS_OK;
  if (!alm || !phase || !workspace) return PS_ERR_INVALID;
  const ps::Plan& P = plan->p;
  if (spin > 0 && !P.d_seed[spin]) return PS_ERR_INVALID;
  if (workspace_bytes < leg_ws_bytes(plan, batch, spin, 0)) return PS_ERR_WORKSPACE;
  const int ncomp = spin == 0 ? 1 : 2;
  double2* almT = static_cast<double2*>(workspace);
  int rc = ps::launch_alm_to_T(reinterpret_cast<const double2*>(alm), almT, batch, ncomp, P.nalm, P.num_sms, stream);
  if (rc) return rc;
  if (P.prec == PS_PREC_MIXED) {
    float2* ph32 = reinterpret_cast<float2*>(static_cast<char*>(workspace) +
                                             align256(size_t(P.nalm) * batch * ncomp * sizeof(double2)));
    TabRef tr;
    if (table_for(plan, spin, tr))
      rc = ps::launch_tab_synth(P, tr.tab, tr.off, tr.Rh_table, tr.toff, almT, ph32, batch, spin, P.d_err, stream,
                                tr.fmt);
    else
      rc = ps::launch_legendre_synth_tc(P, almT, ph32, batch, spin, P.d_err, stream);
    if (rc) return rc;
    const int64_t n = int64_t(P.R) * (P.mmax + 1) * batch * ncomp;
    phase_f32_to_f64<<<convert_grid(n, P.num_sms), 256, 0, stream>>>(ph32, reinterpret_cast<double2*>(phase), n);
    PS_LAUNCH_CHECK();
    return PS_OK;
  }
  return ps::launch_legendre_synth_f64(P, almT, reinterpret_cast<double2*>(phase), batch, spin, stream);
}

int ps_legendre_adjoint(const ps_plan* plan, const double* phase, double* alm, int batch, int spin, double scale,
                        void* workspace, size_t workspace_bytes, cudaStream_t stream) {
  if (!plan || batch < 0 || spin < 0 || spin > 3) return PS_ERR_INVALID;
  if (batch == 0) return PS_OK;
  if (!alm || !phase || !workspace) return PS_ERR_INVALID;
  const ps::Plan& P = plan->p;
  if (spin > 0 && !P.d_seed[spin]) return PS_ERR_INVALID;
  if (workspace_bytes < leg_ws_bytes(plan, batch, spin, 1)) return PS_ERR_WORKSPACE;
  const int ncomp = spin == 0 ? 1 : 2;
  if (P.prec == PS_PREC_MIXED) {
    const int64_t n = int64_t(P.R) * (P.mmax + 1) * batch * ncomp;
    float2* ph32 = static_cast<float2*>(workspace);
    float2* partial = reinterpret_cast<float2*>(static_cast<char*>(workspace) + align256(size_t(n) * sizeof(float2)));
    phase_f64_to_f32<<<convert_grid(n, P.num_sms), 256, 0, stream>>>(reinterpret_cast<const double2*>(phase), ph32, n);
    PS_LAUNCH_CHECK();
    TabRef tr;
    if (table_for(plan, spin, tr))
      return ps::launch_tab_adj(P, tr.tab, tr.off, tr.work, tr.nwork, tr.Rh_table, tr.toff, ph32,
                                reinterpret_cast<double2*>(alm), batch, spin, scale, int64_t(ncomp) * P.nalm, nullptr,
                                P.d_err, stream, tr.fmt);
    const int ch = adjoint_chunk(P, batch, spin);
    for (int b0 = 0; b0 < batch; b0 += ch) {
      const int bc = std::min(ch, batch - b0);
      int rc = ps::launch_legendre_adjoint_mx(P, ph32, partial, batch, b0, bc, spin, stream);
      if (rc) return rc;
      rc = ps::launch_reduce_partials_f32(partial, reinterpret_cast<double2*>(alm), ps::mx_adjoint_tiles(P), bc, ncomp,
                                          P.nalm, scale, b0, P.num_sms, stream);
      if (rc) return rc;
    }
    return PS_OK;
  }
  double2* partial = static_cast<double2*>(workspace);
  const int ch = fp64_adjoint_chunk(batch, spin);
  for (int b0 = 0; b0 < batch; b0 += ch) {
    const int bc = std::min(ch, batch - b0);
    int rc = ps::launch_legendre_adjoint_f64(P, reinterpret_cast<const double2*>(phase), partial, batch, b0, bc,
                                             spin, stream);
    if (rc) return rc;
    rc = ps::launch_reduce_partials(partial, reinterpret_cast<double2*>(alm), ps::adjoint_tiles(P), bc, ncomp,
                                    P.nalm, scale, b0, P.num_sms, stream);
    if (rc) return rc;
  }
  return PS_OK;
}

int ps_sht_workspace_bytes(const ps_plan* plan, int batch, int spin, int adjoint, size_t* bytes) {
  if (!plan || !bytes || batch < 0 || spin < 0 || spin > 3) return PS_ERR_INVALID;
  *bytes = sht_ws_bytes(plan, batch, spin, adjoint);
  return PS_OK;
}

int ps_synthesis(const ps_plan* plan, const double* alm, double* map, int batch, int spin, void* workspace,
                 size_t workspace_bytes, cudaStream_t stream) {
  if (!plan || batch < 0 || spin < 0 || spin > 3) return PS_ERR_INVALID;
  if (plan->is_band) return PS_ERR_UNSUPPORTED;
  if (batch == 0) return PS_OK;
  if (!alm || !map || !workspace) return PS_ERR_INVALID;
  const ps::Plan& P = plan->p;
  if (spin > 0 && !P.d_seed[spin]) return PS_ERR_INVALID;
  if (workspace_bytes < sht_ws_bytes(plan, batch, spin, 0)) return PS_ERR_WORKSPACE;
  const int ncomp = spin == 0 ? 1 : 2;
  const int nf = batch * ncomp;
  char* ws = static_cast<char*>(workspace);
  double2* almT = reinterpret_cast<double2*>(ws);
  char* phase_ptr = ws + align256(size_t(P.nalm) * nf * sizeof(double2));
  int rc;
  if (nf == 1) {
    almT = reinterpret_cast<double2*>(const_cast<double*>(alm));
  } else {
    rc = ps::launch_alm_to_T(reinterpret_cast<const double2*>(alm), almT, batch, ncomp, P.nalm, P.num_sms, stream);
    if (rc) return rc;
  }
  if (P.prec == PS_PREC_MIXED) {
    // tensor-core Legendre stage (TF32 x3, FP32 accumulation) and FP32 ring transforms
    float2* phase = reinterpret_cast<float2*>(phase_ptr);
    TabRef tr;
    if (table_for(plan, spin, tr))
      rc = ps::launch_tab_synth(P, tr.tab, tr.off, tr.Rh_table, tr.toff, almT, phase, batch, spin, P.d_err, stream,
                                tr.fmt);
    else
      rc = ps::launch_legendre_synth_tc(P, almT, phase, batch, spin, P.d_err, stream);
    if (rc) return rc;
    for (size_t c = 0; c < plan->cls_len.size(); ++c) {
      rc = ps::launch_ring_synth_f32(P, plan->d_ring_lists + (spin ? plan->cls_off[c] : plan->cls_off_n[c]),
                                     spin ? plan->cls_cnt[c] : plan->cls_cnt_n[c], plan->cls_len[c], phase, map, nf,
                                     spin > 0, stream);
      if (rc) return rc;
    }
    return PS_OK;
  }
  double2* phase = reinterpret_cast<double2*>(phase_ptr);
  rc = ps::launch_legendre_synth_f64(P, almT, phase, batch, spin, stream);
  if (rc) return rc;
  for (size_t c = 0; c < plan->cls_len.size(); ++c) {
    rc = ps::launch_ring_synth_f64(P, plan->d_ring_lists + (spin ? plan->cls_off[c] : plan->cls_off_n[c]),
                                   spin ? plan->cls_cnt[c] : plan->cls_cnt_n[c], plan->cls_len[c], phase, map, nf,
                                   spin > 0, stream);
    if (rc) return rc;
  }
  return PS_OK;
}

int ps_adjoint(const ps_plan* plan, const double* map, double* alm, int batch, int spin, double scale,
               void* workspace, size_t workspace_bytes, cudaStream_t stream) {
  if (!plan || batch < 0 || spin < 0 || spin > 3) return PS_ERR_INVALID;
  if (plan->is_band) return PS_ERR_UNSUPPORTED;
  if (batch == 0) return PS_OK;
  if (!alm || !map || !workspace) return PS_ERR_INVALID;
  const ps::Plan& P = plan->p;
  if (spin > 0 && !P.d_seed[spin]) return PS_ERR_INVALID;
  if (workspace_bytes < sht_ws_bytes(plan, batch, spin, 1)) return PS_ERR_WORKSPACE;
  const int ncomp = spin == 0 ? 1 : 2;
  const int nf = batch * ncomp;
  char* ws = static_cast<char*>(workspace);
  const size_t phase_bytes = align256(size_t(P.R) * (P.mmax + 1) * nf * sizeof(double2));
  int rc;
  if (P.prec == PS_PREC_MIXED) {
    // FP32 ring transforms, FP64 recurrences with FP32 contractions, FP64 cross-tile sums
    float2* phase = reinterpret_cast<float2*>(ws);
    float2* partial = reinterpret_cast<float2*>(ws + phase_bytes);
    for (size_t c = 0; c < plan->cls_len.size(); ++c) {
      rc = ps::launch_ring_adjoint_f32(P, plan->d_ring_lists + (spin ? plan->cls_off[c] : plan->cls_off_n[c]),
                                       spin ? plan->cls_cnt[c] : plan->cls_cnt_n[c], plan->cls_len[c], map, phase,
                                       nf, spin > 0, stream);
      if (rc) return rc;
    }
    TabRef tr;
    if (table_for(plan, spin, tr))
      return ps::launch_tab_adj(P, tr.tab, tr.off, tr.work, tr.nwork, tr.Rh_table, tr.toff, phase,
                                reinterpret_cast<double2*>(alm), batch, spin, scale, int64_t(ncomp) * P.nalm, nullptr,
                                P.d_err, stream, tr.fmt);
    const int ch = adjoint_chunk(P, batch, spin);
    for (int b0 = 0; b0 < batch; b0 += ch) {
      const int bc = std::min(ch, batch - b0);
      rc = ps::launch_legendre_adjoint_mx(P, phase, partial, batch, b0, bc, spin, stream);
      if (rc) return rc;
      rc = ps::launch_reduce_partials_f32(partial, reinterpret_cast<double2*>(alm), ps::mx_adjoint_tiles(P), bc,
                                          ncomp, P.nalm, scale, b0, P.num_sms, stream);
      if (rc) return rc;
    }
    return PS_OK;
  }
  double2* phase = reinterpret_cast<double2*>(ws);
  double2* partial = reinterpret_cast<double2*>(ws + phase_bytes);
  for (size_t c = 0; c < plan->cls_len.size(); ++c) {
    rc = ps::launch_ring_adjoint_f64(P, plan->d_ring_lists + (spin ? plan->cls_off[c] : plan->cls_off_n[c]),
                                     spin ? plan->cls_cnt[c] : plan->cls_cnt_n[c], plan->cls_len[c], map, phase, nf,
                                     spin > 0, stream);
    if (rc) return rc;
  }
  const int ch = adjoint_chunk(P, batch, spin);
  for (int b0 = 0; b0 < batch; b0 += ch) {
    const int bc = std::min(ch, batch - b0);
    rc = ps::launch_legendre_adjoint_f64(P, phase, partial, batch, b0, bc, spin, stream);
    if (rc) return rc;
    rc = ps::launch_reduce_partials(partial, reinterpret_cast<double2*>(alm), ps::adjoint_tiles(P), bc, ncomp,
                                    P.nalm, scale, b0, P.num_sms, stream);
    if (rc) return rc;
  }
  return PS_OK;
}

}  // extern "C"

namespace ps {
// The pieces of a full mixed-precision plan with the Legendre table of `spin` that the fused
// round trip (ps_roundtrip.cu) needs; PS_ERR_UNSUPPORTED for FP64 or band plans and for spins
// without a table.
struct RoundtripView {
  const Plan* P;
  const float* tab;
  const int64_t* off;
  const int2* work;
  int nwork;
  const int* ring_lists;
  const int* cls_len;
  const int* cls_off;
  const int* cls_cnt;
  const int* cls_off_n;
  const int* cls_cnt_n;
  int ncls;
  int fmt;
};
int roundtrip_view(const ps_plan* plan, int spin, RoundtripView& v) {
  if (plan->is_band || plan->p.prec != PS_PREC_MIXED) return PS_ERR_UNSUPPORTED;
  if (spin > 0 && !plan->p.d_seed[spin]) return PS_ERR_INVALID;
  TabRef tr;
  if (!table_for(plan, spin, tr)) return PS_ERR_UNSUPPORTED;
  v.P = &plan->p;
  v.tab = tr.tab;
  v.off = tr.off;
  v.work = tr.work;
  v.nwork = tr.nwork;
  v.ring_lists = plan->d_ring_lists;
  v.cls_len = plan->cls_len.data();
  v.cls_off = plan->cls_off.data();
  v.cls_cnt = plan->cls_cnt.data();
  v.cls_off_n = plan->cls_off_n.data();
  v.cls_cnt_n = plan->cls_cnt_n.data();
  v.ncls = int(plan->cls_len.size());
  v.fmt = tr.fmt;
  return PS_OK;
}

// The Legendre tables of a mixed band plan (owned by its parent), for the masked-band
// preconditioner (ps_cutprec.cu); PS_ERR_UNSUPPORTED for other plans or a spin without a table.
struct BandView {
  const Plan* P;
  const float* tab;
  const int64_t* off;
  const int2* work;
  int nwork, Rh_table, toff, fmt;
};
int band_view(const ps_plan* band, int spin, BandView& v) {
  if (!band || !band->is_band || band->p.prec != PS_PREC_MIXED) return PS_ERR_UNSUPPORTED;
  if (spin > 0 && !band->p.d_seed[spin]) return PS_ERR_INVALID;
  TabRef tr;
  if (!table_for(band, spin, tr)) return PS_ERR_UNSUPPORTED;
  v.P = &band->p;
  v.tab = tr.tab;
  v.off = tr.off;
  v.work = tr.work;
  v.nwork = tr.nwork;
  v.Rh_table = tr.Rh_table;
  v.toff = tr.toff;
  v.fmt = tr.fmt;
  return PS_OK;
}
}  // namespace ps
