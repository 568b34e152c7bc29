// Launch counters and optional CUDA-event timing of the library's kernels.
//
// Every launcher reports its launches (always counted) and the algorithmic
// work of the launch (flops, bytes).  With timing enabled, a pair of CUDA
// events brackets the launch on its own stream; ps_stats_get synchronises
// those events and sums the durations, so the averages are device times of
// the kernels inside whatever region the caller timed.
#include <mutex>
#include <vector>

#include "ps_common.cuh"
#include "ps_stats.cuh"

namespace ps {
namespace {
struct Acc {
  int64_t launches = 0;
  double flops = 0.0, bytes = 0.0;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev;
};
std::mutex g_mu;
Acc g_acc[PS_KERNEL_KINDS];
bool g_timing = false;
}  // namespace

StatScope::StatScope(int kind, double flops, double bytes, cudaStream_t st) : kind_(kind), st_(st) {
  std::lock_guard<std::mutex> lk(g_mu);
  Acc& a = g_acc[kind];
  a.launches += 1;
  a.flops += flops;
  a.bytes += bytes;
  if (g_timing) {
    cudaEvent_t s, e;
    if (cudaEventCreate(&s) == cudaSuccess && cudaEventCreate(&e) == cudaSuccess) {
      cudaEventRecord(s, st);
      start_ = s;
      stop_ = e;
      timed_ = true;
    }
  }
}

StatScope::~StatScope() {
  if (!timed_) return;
  cudaEventRecord(stop_, st_);
  std::lock_guard<std::mutex> lk(g_mu);
  g_acc[kind_].ev.emplace_back(start_, stop_);
}
}  // namespace ps

extern "C" {

int ps_stats_enable_timing(int on) {
  std::lock_guard<std::mutex> lk(ps::g_mu);
  ps::g_timing = on != 0;
  return PS_OK;
}

int ps_stats_reset(void) {
  std::lock_guard<std::mutex> lk(ps::g_mu);
  for (auto& a : ps::g_acc) {
    for (auto& p : a.ev) { cudaEventDestroy(p.first); cudaEventDestroy(p.second); }
    a = ps::Acc();
  }
  return PS_OK;
}

int ps_stats_get(int kind, int64_t* launches, double* ms, double* flops, double* bytes) {
  if (kind < 0 || kind >= PS_KERNEL_KINDS) return PS_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ps::g_mu);
  ps::Acc& a = ps::g_acc[kind];
  double tot = 0.0;
  for (auto& p : a.ev) {
    if (cudaEventSynchronize(p.second) != cudaSuccess) return PS_ERR_CUDA;
    float t = 0.f;
    if (cudaEventElapsedTime(&t, p.first, p.second) != cudaSuccess) return PS_ERR_CUDA;
    tot += t;
  }
  if (launches) *launches = a.launches;
  if (ms) *ms = tot;
  if (flops) *flops = a.flops;
  if (bytes) *bytes = a.bytes;
  return PS_OK;
}

}  // extern "C"
