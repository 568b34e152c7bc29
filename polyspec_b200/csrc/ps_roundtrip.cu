// Weighted synthesis-adjoint round trip of the masked CG's operator, fused:
//   alm_out = lscale * scale * Y^H W Y (lscale * alm_in)
// per spin, with Y the synthesis, W a per-pixel weight of each map component and
// lscale an optional per-(component, lm) factor (the beam).  For a mixed-precision
// plan holding the Legendre table of the spin this runs as: strided gather of the
// input alm with the factor (layout [nalm][batch][ncomp]) -> table synthesis
// (tensor cores) -> one ring kernel per FFT length class that synthesises each
// ring in shared memory, weights its pixels and transforms it back (the maps
// never reach HBM) -> table adjoint writing the strided output with the factor.
// Without the table the entry returns PS_ERR_UNSUPPORTED and the caller composes
// ps_synthesis, the weighting and ps_adjoint itself.
#include <algorithm>

#include "ps_common.cuh"
#include "ps_stats.cuh"

struct ps_plan;

namespace ps {
int launch_tab_synth(const Plan& P, const float* table, const int64_t* d_blockoff, int Rh_table, int toff,
                     const double2* almT, float2* phase, int B, int spin, int* err_flag, cudaStream_t st, int fmt);
int launch_tab_adj(const Plan& P, const float* table, const int64_t* d_blockoff, const int2* d_work, int nwork,
                   int Rh_table, int toff, const float2* phase, double2* alm, int B, int spin, double scale,
                   int64_t out_stride, const double* lscale, int* err_flag, cudaStream_t st, int fmt);
int launch_ring_roundtrip_f32(const Plan& P, const int* d_list, int nrings, int work_len, float2* phase,
                              const double* weight, int nf, int pack, cudaStream_t st);

namespace {
// alm (B maps at stride `stride` complex elements, ncomp components of nalm each) times
// lscale[comp][idx] (when given) -> almT [nalm][B][ncomp]
__global__ void alm_gather_scaled(const double2* __restrict__ alm, int64_t stride, const double* __restrict__ lscale,
                                  double2* __restrict__ almT, int B, int ncomp, int64_t nalm) {
  const int64_t n = nalm * B * ncomp;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < n; t += int64_t(gridDim.x) * blockDim.x) {
    const int c = int(t % ncomp);
    const int b = int((t / ncomp) % B);
    const int64_t idx = t / (int64_t(ncomp) * B);
    double2 v = alm[int64_t(b) * stride + int64_t(c) * nalm + idx];
    if (lscale) {
      const double f = lscale[int64_t(c) * nalm + idx];
      v.x *= f;
      v.y *= f;
    }
    almT[t] = v;
  }
}
size_t al256(size_t x) { return (x + 255) & ~size_t(255); }
}  // namespace

// the pieces of a plan the round trip needs, resolved by the plan code (ps_plan.cu)
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
int roundtrip_view(const ps_plan* plan, int spin, RoundtripView& v);

}  // namespace ps

extern "C" int ps_roundtrip_workspace_bytes(const ps_plan* plan, int batch, int spin, size_t* bytes) {
  if (!plan || !bytes || batch < 0 || spin < 0 || spin > 3) return PS_ERR_INVALID;
  ps::RoundtripView v;
  const int rc = ps::roundtrip_view(plan, spin, v);
  if (rc != PS_OK) return rc;
  const ps::Plan& P = *v.P;
  const size_t nf = size_t(batch) * (spin == 0 ? 1 : 2);
  *bytes = ps::al256(size_t(P.nalm) * nf * sizeof(double2)) + ps::al256(size_t(P.R) * (P.mmax + 1) * nf * sizeof(float2));
  return PS_OK;
}

extern "C" int ps_sht_weighted_roundtrip(const ps_plan* plan, const double* alm_in, double* alm_out,
                                         int64_t alm_stride, int batch, int spin, const double* weight,
                                         const double* lscale, double scale, void* workspace,
                                         size_t workspace_bytes, cudaStream_t stream) {
  if (!plan || batch < 0 || spin < 0 || spin > 3) return PS_ERR_INVALID;
  if (batch == 0) return PS_OK;
  ps::RoundtripView v;
  int rc = ps::roundtrip_view(plan, spin, v);
  if (rc != PS_OK) return rc;
  const ps::Plan& P = *v.P;
  const int ncomp = spin == 0 ? 1 : 2;
  if (!alm_in || !alm_out || !weight || !workspace || alm_stride < int64_t(ncomp) * P.nalm) return PS_ERR_INVALID;
  size_t need = 0;
  rc = ps_roundtrip_workspace_bytes(plan, batch, spin, &need);
  if (rc != PS_OK) return rc;
  if (workspace_bytes < need) return PS_ERR_WORKSPACE;
  const int nf = batch * ncomp;
  char* ws = static_cast<char*>(workspace);
  double2* almT = reinterpret_cast<double2*>(ws);
  float2* phase = reinterpret_cast<float2*>(ws + ps::al256(size_t(P.nalm) * nf * sizeof(double2)));
  {
    const int64_t n = P.nalm * int64_t(nf);
    int blocks = int(std::min<int64_t>((n + 255) / 256, int64_t(P.num_sms) * 8));
    if (blocks < 1) blocks = 1;
    ps::StatScope sc(PS_K_LAYOUT, 0.0, 32.0 * n, stream);
    ps::alm_gather_scaled<<<blocks, 256, 0, stream>>>(reinterpret_cast<const double2*>(alm_in), alm_stride, lscale,
                                                      almT, batch, ncomp, P.nalm);
    PS_LAUNCH_CHECK();
  }
  rc = ps::launch_tab_synth(P, v.tab, v.off, P.Rh, 0, almT, phase, batch, spin, P.d_err, stream, v.fmt);
  if (rc) return rc;
  for (int c = 0; c < v.ncls; ++c) {
    rc = ps::launch_ring_roundtrip_f32(P, v.ring_lists + (spin ? v.cls_off[c] : v.cls_off_n[c]),
                                       spin ? v.cls_cnt[c] : v.cls_cnt_n[c], v.cls_len[c], phase, weight, nf,
                                       spin > 0, stream);
    if (rc) return rc;
  }
  return ps::launch_tab_adj(P, v.tab, v.off, v.work, v.nwork, P.Rh, 0, phase, reinterpret_cast<double2*>(alm_out),
                            batch, spin, scale, alm_stride, lscale, P.d_err, stream, v.fmt);
}
