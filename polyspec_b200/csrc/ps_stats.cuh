// Launch accounting of libpscuda (see ps_stats.cu).
#pragma once
#include <cuda_runtime.h>

namespace ps {
// RAII scope around one kernel launch: counts it, adds its algorithmic work
// and, when timing is enabled, records CUDA events around it on `st`.
class StatScope {
 public:
  StatScope(int kind, double flops, double bytes, cudaStream_t st);
  ~StatScope();
  StatScope(const StatScope&) = delete;
  StatScope& operator=(const StatScope&) = delete;

 private:
  int kind_;
  cudaStream_t st_;
  cudaEvent_t start_{}, stop_{};
  bool timed_ = false;
};
}  // namespace ps
