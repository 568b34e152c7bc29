// Allocation-free spherical-harmonic synthesis.
//
// Some callers cannot allocate device memory when they need a transform: code
// that runs inside a framework which owns all device memory through its own
// fixed-budget allocator, or a real-time loop in which a cudaMalloc (which may
// synchronise the device) is not allowed.  For them ps_synthesis_noalloc takes
// the scratch that ps_synthesis would take from the caller's workspace from a
// file-scope static device array instead, so the call itself allocates nothing.
// The plan must still be created beforehand with ps_plan_create (that call does
// allocate its read-only tables).
//
// The array is PS_NOALLOC_SCRATCH_BYTES (16 MiB) and every GPU that loads this
// library keeps it until the process exits.  All calls on a device share it and
// it keeps the last call's contents; nothing in it needs to start at zero
// (the transposed alm and the per-ring phases are fully rewritten by every
// call), but two calls whose kernels overlap on the GPU -- on different streams,
// or from different host threads -- race on it.
#include <mutex>

#include "ps_common.cuh"

namespace {

// In host code this name is only a host-side stand-in for the device array:
// its device address comes from cudaGetSymbolAddress below, once per device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[PS_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_addr[kMaxDevices] = {};

// Device address of the scratch array on the current device; looked up on the
// first call per device (so that first call should come before any stream
// capture) and cached.
int scratch_address(void** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return PS_ERR_CUDA;
  if (dev < 0 || dev >= kMaxDevices) return PS_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || p == nullptr) return PS_ERR_CUDA;
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return PS_OK;
}

}  // namespace

extern "C" int ps_synthesis_noalloc(const ps_plan* plan, const double* alm, double* map, int batch, int spin,
                                    cudaStream_t stream) {
  if (!plan || batch < 0 || spin < 0 || spin > 3) return PS_ERR_INVALID;
  if (batch == 0) return PS_OK;
  if (!alm || !map) return PS_ERR_INVALID;
  size_t need = 0;
  int rc = ps_sht_workspace_bytes(plan, batch, spin, 0, &need);
  if (rc != PS_OK) return rc;
  if (need > size_t(PS_NOALLOC_SCRATCH_BYTES)) return PS_ERR_WORKSPACE;  // larger than the static scratch
  void* scratch = nullptr;
  rc = scratch_address(&scratch);
  if (rc != PS_OK) return rc;
  return ps_synthesis(plan, alm, map, batch, spin, scratch, size_t(PS_NOALLOC_SCRATCH_BYTES), stream);
}
