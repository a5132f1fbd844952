// b2_profile.cuh -- RAII scope placed around every kernel launch: counts the
// launch and, when per-thread profiling is on, brackets it with CUDA events
// recorded on the launch stream.
#pragma once
#include <cuda_runtime.h>

namespace b2 {
class ProfScope {
 public:
  ProfScope(const char *name, cudaStream_t s);
  ~ProfScope();
  ProfScope(const ProfScope &) = delete;
  ProfScope &operator=(const ProfScope &) = delete;

 private:
  const char *name_;
  cudaStream_t s_;
  void *a_ = nullptr;
};
}  // namespace b2

#define B2_PROF(name, stream) ::b2::ProfScope _b2_prof_scope(name, stream)
