// Per-kernel CUDA-event timing (see profile.cu).  Usage inside a host function:
//   { HS2_PROF("ba_schur", stream); kernel<<<..., stream>>>(...); }
#pragma once

#include <cuda_runtime.h>

namespace hs2 {

class ProfScope {
 public:
  ProfScope(const char* name, cudaStream_t s);
  ~ProfScope();
  ProfScope(const ProfScope&) = delete;
  ProfScope& operator=(const ProfScope&) = delete;

 private:
  const char* name_;
  cudaStream_t stream_;
  cudaEvent_t start_;
};

}  // namespace hs2

#define HS2_PROF_CAT2(a, b) a##b
#define HS2_PROF_CAT(a, b) HS2_PROF_CAT2(a, b)
#define HS2_PROF(name, stream) ::hs2::ProfScope HS2_PROF_CAT(hs2_prof_, __LINE__)(name, stream)
