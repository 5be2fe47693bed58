// Error reporting and device binding shared by every entry point.
#include <atomic>
#include <cstdarg>
#include <cstdio>

#include "common.cuh"

namespace hs2 {

static thread_local char g_last_error[512] = "";
static std::atomic<long long> g_launches{0};

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
}

int cuda_status(cudaError_t e, const char* what) {
  set_error("%s: %s", what, cudaGetErrorString(e));
  return HS2_ERR_CUDA;
}

int bind_device(const void* ptr) {
  if (ptr == nullptr) return HS2_OK;
  cudaPointerAttributes attr;
  cudaError_t e = cudaPointerGetAttributes(&attr, ptr);
  if (e != cudaSuccess) return cuda_status(e, "cudaPointerGetAttributes");
  if (attr.type != cudaMemoryTypeDevice && attr.type != cudaMemoryTypeManaged) {
    set_error("expected a device pointer (got memory type %d)", (int)attr.type);
    return HS2_ERR_INVALID;
  }
  int cur = -1;
  e = cudaGetDevice(&cur);
  if (e != cudaSuccess) return cuda_status(e, "cudaGetDevice");
  if (cur != attr.device) {
    e = cudaSetDevice(attr.device);
    if (e != cudaSuccess) return cuda_status(e, "cudaSetDevice");
  }
  return HS2_OK;
}

}  // namespace hs2

extern "C" const char* hs2_last_error(void) { return hs2::g_last_error; }

extern "C" int hs2_version(void) { return (1 << 16) | 0; }

extern "C" long long hs2_launch_count(void) { return hs2::g_launches.load(std::memory_order_relaxed); }
