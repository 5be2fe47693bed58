// Shared device helpers for the hislam2_b200 kernels (sm_100a).
//
// SE3 conventions follow the reference operator surface: a pose is
// [tx, ty, tz, qx, qy, qz, qw] (HI-SLAM2 hislam2/depth_video.py:43), a tangent
// vector is [tau(3), phi(3)], and the relative pose of an edge i->j is
// Gij = Gj * Gi^-1 (src/droid_kernels.cu:148-159).
#pragma once

#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include <atomic>
#include <mutex>
#include <type_traits>

#include "hislam2_b200.h"

namespace hs2 {

constexpr float kMinDepth = 0.25f;   // points closer than this are dropped (droid_kernels.cu:26)
constexpr int kNumSMs = 148;         // B200

// ---------------------------------------------------------------- status ---
void set_error(const char* fmt, ...);
int cuda_status(cudaError_t e, const char* what);
void count_launch();

#define HS2_CUDA(call)                                                   \
  do {                                                                   \
    cudaError_t e_ = (call);                                             \
    if (e_ != cudaSuccess) return ::hs2::cuda_status(e_, #call);         \
  } while (0)

// Checks the launch that precedes it and counts it (hs2_launch_count()).
#define HS2_LAUNCH_CHECK(name)                                           \
  do {                                                                   \
    ::hs2::count_launch();                                               \
    cudaError_t e_ = cudaGetLastError();                                 \
    if (e_ != cudaSuccess) return ::hs2::cuda_status(e_, name);          \
  } while (0)

// Makes the device that owns `ptr` current for this thread (a no-op when it
// already is).  All entry points take device pointers from the caller.
int bind_device(const void* ptr);

// One-time per-device set-up (kernel attributes, occupancy queries) that any
// host thread may trigger.  `run(dev)` executes `fn` at most once per device
// ordinal that succeeds, under a mutex; ordinals >= kMaxDevices are refused.
constexpr int kMaxDevices = 64;
struct DeviceOnce {
  std::atomic<bool> done[kMaxDevices] = {};
  std::mutex mu;
  template <typename F>
  int run(int dev, F&& fn) {
    if (dev < 0 || dev >= kMaxDevices) {
      set_error("device ordinal %d out of range (at most %d devices)", dev, kMaxDevices);
      return HS2_ERR_INVALID;
    }
    if (done[dev].load(std::memory_order_acquire)) return HS2_OK;
    std::lock_guard<std::mutex> lk(mu);
    if (done[dev].load(std::memory_order_relaxed)) return HS2_OK;
    const int rc = fn();
    if (rc == HS2_OK) done[dev].store(true, std::memory_order_release);
    return rc;
  }
};

// ----------------------------------------------------------- conversions ---
template <typename T> __device__ __forceinline__ float to_f(T v);
template <> __device__ __forceinline__ float to_f<float>(float v) { return v; }
template <> __device__ __forceinline__ float to_f<double>(double v) { return (float)v; }
template <> __device__ __forceinline__ float to_f<__half>(__half v) { return __half2float(v); }
template <> __device__ __forceinline__ float to_f<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }

template <typename T> __device__ __forceinline__ T from_f(float v);
template <> __device__ __forceinline__ float from_f<float>(float v) { return v; }
template <> __device__ __forceinline__ double from_f<double>(float v) { return (double)v; }
template <> __device__ __forceinline__ __half from_f<__half>(float v) { return __float2half_rn(v); }
template <> __device__ __forceinline__ __nv_bfloat16 from_f<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }

// ----------------------------------------------------------- reductions ---
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// ----------------------------------------------------------------- SE3 ---
// Rotation of a 3-vector by a unit quaternion: X + 2w (v x X) + 2 v x (v x X).
template <typename S>
__device__ __forceinline__ void quat_rotate(const S* q, const S* X, S* Y) {
  S c0 = S(2) * (q[1] * X[2] - q[2] * X[1]);
  S c1 = S(2) * (q[2] * X[0] - q[0] * X[2]);
  S c2 = S(2) * (q[0] * X[1] - q[1] * X[0]);
  Y[0] = X[0] + q[3] * c0 + (q[1] * c2 - q[2] * c1);
  Y[1] = X[1] + q[3] * c1 + (q[2] * c0 - q[0] * c2);
  Y[2] = X[2] + q[3] * c2 + (q[0] * c1 - q[1] * c0);
}

// Gij = Gj * Gi^-1 for poses (ti, qi), (tj, qj).
template <typename S>
__device__ __forceinline__ void relative_pose(const S* ti, const S* qi, const S* tj, const S* qj,
                                              S* tij, S* qij) {
  // qij = qj (x) conj(qi)
  qij[0] = qi[3] * qj[0] - qj[3] * qi[0] + (qj[2] * qi[1] - qj[1] * qi[2]);
  qij[1] = qi[3] * qj[1] - qj[3] * qi[1] + (qj[0] * qi[2] - qj[2] * qi[0]);
  qij[2] = qi[3] * qj[2] - qj[3] * qi[2] + (qj[1] * qi[0] - qj[0] * qi[1]);
  qij[3] = qj[3] * qi[3] + qj[0] * qi[0] + qj[1] * qi[1] + qj[2] * qi[2];
  S r[3];
  quat_rotate(qij, ti, r);
  tij[0] = tj[0] - r[0];
  tij[1] = tj[1] - r[1];
  tij[2] = tj[2] - r[2];
}

// Maps a point Jacobian row Jj (w.r.t. a left perturbation of Gj) to the one
// w.r.t. Gi: Ji = -Adj(Gij)^T Jj.  With R = R(qij) and t = tij:
//   Ji[0:3] = -R^T Jj[0:3]
//   Ji[3:6] = -R^T (Jj[3:6] + Jj[0:3] x t)
template <typename S>
__device__ __forceinline__ void pose_jacobian_i(const S* tij, const S* qij, const S* Jj, S* Ji) {
  S qinv[4] = {-qij[0], -qij[1], -qij[2], qij[3]};
  S a[3] = {Jj[0], Jj[1], Jj[2]};
  S m[3] = {Jj[3] + (a[1] * tij[2] - a[2] * tij[1]),
            Jj[4] + (a[2] * tij[0] - a[0] * tij[2]),
            Jj[5] + (a[0] * tij[1] - a[1] * tij[0])};
  S r0[3], r1[3];
  quat_rotate(qinv, a, r0);
  quat_rotate(qinv, m, r1);
  Ji[0] = -r0[0]; Ji[1] = -r0[1]; Ji[2] = -r0[2];
  Ji[3] = -r1[0]; Ji[4] = -r1[1]; Ji[5] = -r1[2];
}

// Left retraction (t, q) <- exp(xi) * (t, q), computed in double precision.
// exp uses the closed-form SO3/SE3 series with Taylor branches for small angles.
__device__ __forceinline__ void retract_left(const double* xi, double* t, double* q) {
  const double* tau = xi;
  const double* phi = xi + 3;
  double th2 = phi[0] * phi[0] + phi[1] * phi[1] + phi[2] * phi[2];
  double th = sqrt(th2);
  double s_half, c_half;
  if (th2 < 1e-8) {
    s_half = 0.5 - th2 / 48.0 + th2 * th2 / 3840.0;
    c_half = 1.0 - th2 / 8.0 + th2 * th2 / 384.0;
  } else {
    s_half = sin(0.5 * th) / th;
    c_half = cos(0.5 * th);
  }
  double dq[4] = {s_half * phi[0], s_half * phi[1], s_half * phi[2], c_half};
  // V * tau with V = I + a [phi]x + b [phi]x^2
  double c1[3] = {phi[1] * tau[2] - phi[2] * tau[1], phi[2] * tau[0] - phi[0] * tau[2],
                  phi[0] * tau[1] - phi[1] * tau[0]};
  double c2[3] = {phi[1] * c1[2] - phi[2] * c1[1], phi[2] * c1[0] - phi[0] * c1[2],
                  phi[0] * c1[1] - phi[1] * c1[0]};
  double dt[3] = {tau[0], tau[1], tau[2]};
  if (th > 1e-4) {
    double a = (1.0 - cos(th)) / th2;
    double b = (th - sin(th)) / (th * th2);
    for (int k = 0; k < 3; ++k) dt[k] += a * c1[k] + b * c2[k];
  }
  double q1[4];
  q1[0] = dq[3] * q[0] + q[3] * dq[0] + (dq[1] * q[2] - dq[2] * q[1]);
  q1[1] = dq[3] * q[1] + q[3] * dq[1] + (dq[2] * q[0] - dq[0] * q[2]);
  q1[2] = dq[3] * q[2] + q[3] * dq[2] + (dq[0] * q[1] - dq[1] * q[0]);
  q1[3] = dq[3] * q[3] - (dq[0] * q[0] + dq[1] * q[1] + dq[2] * q[2]);
  double tr[3];
  quat_rotate(dq, t, tr);
  for (int k = 0; k < 3; ++k) t[k] = tr[k] + dt[k];
  for (int k = 0; k < 4; ++k) q[k] = q1[k];
}

}  // namespace hs2
