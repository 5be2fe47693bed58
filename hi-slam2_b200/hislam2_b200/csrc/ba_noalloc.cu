// hs2_ba_noalloc: bundle adjustment that allocates nothing.
//
// Some callers cannot allocate device memory at the moment they run a BA step:
// a real-time process that fixes its GPU memory budget at start-up, or a host in
// another language that has no caching allocator and cannot afford the
// device-wide synchronisation of cudaMalloc / cudaFree in its tracking loop.  For
// them this entry point takes its scratch from one static device array of this file
// instead of a caller workspace.
//
// The array is sized for a frontend window (kNoAllocScratchBytes = 64 MiB,
// enough for e.g. 25 keyframes and ~300 edges on a 43x77 grid); every GPU that
// loads this part of the library holds it until the process exits.  Problems
// whose workspace is larger are rejected.  All calls share the array: a call
// overwrites what the previous one left there (hs2_ba clears everything it needs
// to start from zero), and calls whose GPU work overlaps in time -- on two
// streams, or from two threads -- race on it and must be serialised by the caller.
#include <mutex>

#include "common.cuh"

namespace hs2 {

constexpr size_t kNoAllocScratchBytes = size_t(64) << 20;
constexpr int kNoAllocMaxDevices = 64;

// Device-side scratch.  In host code this name is only a stand-in for the
// symbol: its device address is obtained with cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_ba_scratch[kNoAllocScratchBytes];

static std::mutex g_scratch_mu;
static void* g_scratch_addr[kNoAllocMaxDevices] = {nullptr};

// Device address of g_ba_scratch on the current device; looked up once per device
// (the first call on a device does this set-up).
static int scratch_address(void** out) {
  int dev = 0;
  HS2_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoAllocMaxDevices) {
    set_error("ba_noalloc: device ordinal %d out of range", dev);
    return HS2_ERR_INVALID;
  }
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (g_scratch_addr[dev] == nullptr) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_ba_scratch);
    if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(g_ba_scratch)");
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return HS2_OK;
}

}  // namespace hs2

extern "C" int hs2_ba_noalloc(float* poses, int64_t num_poses, float* disps, int64_t num_disps, int ht, int wd,
                              const float* intrinsics, const float* targets, const float* weights,
                              const float* eta, int64_t eta_rows, const int64_t* ii, const int64_t* jj,
                              int64_t num_edges, int t0, int t1, int iterations, float lm, float ep,
                              int motion_only, float* dx, float* dz, int64_t dz_rows, int32_t* info,
                              hs2_stream_t stream) {
  using namespace hs2;
  size_t need = 0;
  int rc = hs2_ba_workspace_size(num_poses, num_disps, ht, wd, num_edges, t0, t1, motion_only, &need);
  if (rc) return rc;
  if (need > kNoAllocScratchBytes) {
    set_error("ba_noalloc: this problem needs %zu bytes of scratch; the allocation-free entry point has %zu "
              "(use hs2_ba with a caller workspace)", need, kNoAllocScratchBytes);
    return HS2_ERR_WORKSPACE;
  }
  if ((rc = bind_device(poses))) return rc;
  void* scratch = nullptr;
  if ((rc = scratch_address(&scratch))) return rc;
  return hs2_ba(poses, num_poses, disps, num_disps, ht, wd, intrinsics, targets, weights, eta, eta_rows, ii, jj,
                num_edges, t0, t1, iterations, lm, ep, motion_only, dx, dz, dz_rows, info, scratch,
                kNoAllocScratchBytes, stream);
}
