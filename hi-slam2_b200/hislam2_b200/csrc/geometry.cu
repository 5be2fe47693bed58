// iproj / covis_distance / depth_filter: the per-pixel back-projection helpers of the
// keyframe policy and of the point-cloud filter (reference: src/droid_kernels.cu
// covis_distance_kernel :996-1090, depth_filter_kernel :1094-1204, iproj_kernel
// :1208-1272, host wrappers :2071-2143).
//
// All three are one pass over disparity planes; the pose algebra matches the reference's
// actSO3/relSE3 operation order (quat_rotate, relative_pose).
//   iproj           thread per pixel of frame b: (R_b X + d t_b) / d, stored as [N,H,W,3].
//   covis_distance  CTA per entry: count of frame i's pixels outside the image under
//                   both G(i-1) Gi^-1 and G(i+1) Gi^-1, divided by H*W.
//   depth_filter    thread per (entry, neighbour, pixel) with the reference's neighbour
//                   set {i-1, i-2, i-3, i+3, i+4, i+5}; +1 in counter[b] when the
//                   reprojected inverse depth is within thresh[b] of one of the four
//                   disparities around the reprojection (compared in double precision,
//                   as the reference's 1.0/dj does).  Counts are small integers, so the
//                   atomic sum is order-independent.
// Entries whose frame index lies outside the buffers (the reference reads out of bounds
// there) set HS2_DEV_BAD_INDEX and produce no output for that entry.
#include "common.cuh"
#include "profile.cuh"

namespace hs2 {

constexpr int kGeoThreads = 256;

__global__ void __launch_bounds__(kGeoThreads)
iproj_kernel(const float* __restrict__ poses, const float* __restrict__ disps, int ht, int wd,
             const float* __restrict__ intr, float* __restrict__ points) {
  const int b = blockIdx.y;
  const int HW = ht * wd;
  const int k = blockIdx.x * kGeoThreads + threadIdx.x;
  if (k >= HW) return;
  const float fx = intr[0], fy = intr[1], cx = intr[2], cy = intr[3];
  const float* t = poses + 7 * (int64_t)b;
  const float q[4] = {t[3], t[4], t[5], t[6]};
  const int vi = k / wd;
  const float u = (float)(k - vi * wd), v = (float)vi;
  const float X[3] = {(u - cx) / fx, (v - cy) / fy, 1.0f};
  const float d = disps[(int64_t)b * HW + k];
  float Y[3];
  quat_rotate(q, X, Y);
  float* o = points + ((int64_t)b * HW + k) * 3;
  o[0] = (Y[0] + d * t[0]) / d;
  o[1] = (Y[1] + d * t[1]) / d;
  o[2] = (Y[2] + d * t[2]) / d;
}

__global__ void __launch_bounds__(kGeoThreads)
covis_distance_kernel(const float* __restrict__ poses, int64_t num_poses, const float* __restrict__ disps,
                      int64_t num_disps, int ht, int wd, const float* __restrict__ intr,
                      const int64_t* __restrict__ ii, float* __restrict__ dist, int32_t* __restrict__ info) {
  const int n = blockIdx.x;
  const int64_t i = ii[n];
  if (i < 1 || i + 1 >= num_poses || i >= num_disps) {
    if (threadIdx.x == 0) {
      dist[n] = 0.f;
      atomicOr(info, HS2_DEV_BAD_INDEX);
    }
    return;
  }
  const float fx = intr[0], fy = intr[1], cx = intr[2], cy = intr[3];
  float t1[3], q1[4], t2[3], q2[4];
  relative_pose(poses + 7 * i, poses + 7 * i + 3, poses + 7 * (i - 1), poses + 7 * (i - 1) + 3, t1, q1);
  relative_pose(poses + 7 * i, poses + 7 * i + 3, poses + 7 * (i + 1), poses + 7 * (i + 1) + 3, t2, q2);
  const int HW = ht * wd;
  const float* drow = disps + i * HW;
  int count = 0;
  for (int k = threadIdx.x; k < HW; k += kGeoThreads) {
    const int vi = k / wd;
    const float u = (float)(k - vi * wd), v = (float)vi;
    const float X[3] = {(u - cx) / fx, (v - cy) / fy, 1.0f};
    const float d = drow[k];
    float Y1[3], Y2[3];
    quat_rotate(q1, X, Y1);
    quat_rotate(q2, X, Y2);
    Y1[0] += d * t1[0]; Y1[1] += d * t1[1]; Y1[2] += d * t1[2];
    Y2[0] += d * t2[0]; Y2[1] += d * t2[1]; Y2[2] += d * t2[2];
    const float x1 = fx * (Y1[0] / Y1[2]) + cx, y1 = fy * (Y1[1] / Y1[2]) + cy;
    const float x2 = fx * (Y2[0] / Y2[2]) + cx, y2 = fy * (Y2[1] / Y2[2]) + cy;
    const bool out1 = x1 < 0 || x1 >= wd || y1 < 0 || y1 >= ht;
    const bool out2 = x2 < 0 || x2 >= wd || y2 < 0 || y2 >= ht;
    count += (out1 && out2) ? 1 : 0;
  }
  __shared__ int red[kGeoThreads / 32];
  count = __reduce_add_sync(0xffffffffu, count);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = count;
  __syncthreads();
  if (threadIdx.x == 0) {
    int tot = 0;
    for (int w = 0; w < kGeoThreads / 32; ++w) tot += red[w];
    dist[n] = (float)tot / (float)HW;
  }
}

__global__ void __launch_bounds__(kGeoThreads)
depth_filter_kernel(const float* __restrict__ poses, const float* __restrict__ disps, int64_t num_disps, int ht,
                    int wd, const float* __restrict__ intr, const int64_t* __restrict__ ix,
                    const float* __restrict__ thresh, float* __restrict__ counter, int32_t* __restrict__ info) {
  const int b = blockIdx.x, nb = blockIdx.y;
  const int HW = ht * wd;
  const int k = blockIdx.z * kGeoThreads + threadIdx.x;
  const int64_t i = ix[b];
  if (i < 0 || i >= num_disps) {
    if (nb == 0 && blockIdx.z == 0 && threadIdx.x == 0) atomicOr(info, HS2_DEV_BAD_INDEX);
    return;
  }
  const int64_t j = nb < 3 ? i - nb - 1 : i + nb;
  if (j < 0 || j >= num_disps || k >= HW) return;
  const float fx = intr[0], fy = intr[1], cx = intr[2], cy = intr[3];
  float tij[3], qij[4];
  relative_pose(poses + 7 * i, poses + 7 * i + 3, poses + 7 * j, poses + 7 * j + 3, tij, qij);
  const int vi = k / wd;
  const float u = (float)(k - vi * wd), v = (float)vi;
  const float X[3] = {(u - cx) / fx, (v - cy) / fy, 1.0f};
  const float d = disps[i * HW + k];
  float Y[3];
  quat_rotate(qij, X, Y);
  Y[0] += d * tij[0]; Y[1] += d * tij[1]; Y[2] += d * tij[2];
  const float uj = fx * (Y[0] / Y[2]) + cx;
  const float vj = fy * (Y[1] / Y[2]) + cy;
  const float dj = d / Y[2];
  const int u0 = (int)floorf(uj), v0 = (int)floorf(vj);
  if (u0 >= 0 && v0 >= 0 && u0 < wd - 1 && v0 < ht - 1) {
    const float* dr = disps + j * HW;
    const double t = (double)thresh[b];
    const double inv = 1.0 / (double)dj;
    const float d00 = dr[v0 * wd + u0], d01 = dr[v0 * wd + u0 + 1];
    const float d10 = dr[(v0 + 1) * wd + u0], d11 = dr[(v0 + 1) * wd + u0 + 1];
    if (fabs(inv - 1.0 / (double)d00) < t || fabs(inv - 1.0 / (double)d01) < t ||
        fabs(inv - 1.0 / (double)d10) < t || fabs(inv - 1.0 / (double)d11) < t)
      atomicAdd(&counter[(int64_t)b * HW + k], 1.0f);
  }
}

static int check_geo(const char* op, int64_t num_poses, int64_t num_disps, int ht, int wd) {
  if (num_poses < 0 || num_disps < 0 || ht <= 0 || wd <= 0 || (int64_t)ht * wd > (1 << 30)) {
    set_error("%s: bad sizes num_poses=%lld num_disps=%lld ht=%d wd=%d", op, (long long)num_poses,
              (long long)num_disps, ht, wd);
    return HS2_ERR_INVALID;
  }
  return HS2_OK;
}

}  // namespace hs2

extern "C" int hs2_iproj(const float* poses, int64_t num_poses, const float* disps, int64_t num_disps, int ht, int wd,
                         const float* intrinsics, float* points, hs2_stream_t stream) {
  using namespace hs2;
  int rc = check_geo("iproj", num_poses, num_disps, ht, wd);
  if (rc) return rc;
  if (num_poses < num_disps) {
    set_error("iproj: poses (%lld) must cover every disparity frame (%lld)", (long long)num_poses,
              (long long)num_disps);
    return HS2_ERR_INVALID;
  }
  if (num_disps == 0) return HS2_OK;
  if ((rc = bind_device(points))) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  const int HW = ht * wd;
  if (num_disps > 65535) {
    set_error("iproj: %lld frames exceed the launch grid", (long long)num_disps);
    return HS2_ERR_INVALID;
  }
  HS2_PROF("iproj", s);
  iproj_kernel<<<dim3((HW + kGeoThreads - 1) / kGeoThreads, (unsigned)num_disps), kGeoThreads, 0, s>>>(
      poses, disps, ht, wd, intrinsics, points);
  HS2_LAUNCH_CHECK("iproj_kernel");
  return HS2_OK;
}

extern "C" int hs2_covis_distance(const float* poses, int64_t num_poses, const float* disps, int64_t num_disps,
                                  int ht, int wd, const float* intrinsics, const int64_t* ii, int64_t num,
                                  float* dist, int32_t* info, hs2_stream_t stream) {
  using namespace hs2;
  int rc = check_geo("covis_distance", num_poses, num_disps, ht, wd);
  if (rc) return rc;
  if (num < 0 || num > 0x7fffffff) {
    set_error("covis_distance: bad entry count %lld", (long long)num);
    return HS2_ERR_INVALID;
  }
  if (num == 0) return HS2_OK;
  if ((rc = bind_device(dist))) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  HS2_PROF("covis_distance", s);
  covis_distance_kernel<<<(unsigned)num, kGeoThreads, 0, s>>>(poses, num_poses, disps, num_disps, ht, wd,
                                                              intrinsics, ii, dist, info);
  HS2_LAUNCH_CHECK("covis_distance_kernel");
  return HS2_OK;
}

extern "C" int hs2_depth_filter(const float* poses, int64_t num_poses, const float* disps, int64_t num_disps, int ht,
                                int wd, const float* intrinsics, const int64_t* ix, const float* thresh,
                                int64_t num, float* counter, int32_t* info, hs2_stream_t stream) {
  using namespace hs2;
  int rc = check_geo("depth_filter", num_poses, num_disps, ht, wd);
  if (rc) return rc;
  if (num_poses < num_disps) {
    set_error("depth_filter: poses (%lld) must cover every disparity frame (%lld)", (long long)num_poses,
              (long long)num_disps);
    return HS2_ERR_INVALID;
  }
  if (num < 0 || num > 0x7fffffff) {
    set_error("depth_filter: bad entry count %lld", (long long)num);
    return HS2_ERR_INVALID;
  }
  if (num == 0) return HS2_OK;
  if ((rc = bind_device(counter))) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  const int HW = ht * wd;
  if ((HW + kGeoThreads - 1) / kGeoThreads > 65535) {
    set_error("depth_filter: %d pixels per frame exceed the launch grid", HW);
    return HS2_ERR_INVALID;
  }
  HS2_CUDA(cudaMemsetAsync(counter, 0, sizeof(float) * (size_t)num * HW, s));
  HS2_PROF("depth_filter", s);
  depth_filter_kernel<<<dim3((unsigned)num, 6, (HW + kGeoThreads - 1) / kGeoThreads), kGeoThreads, 0, s>>>(
      poses, disps, num_disps, ht, wd, intrinsics, ix, thresh, counter, info);
  HS2_LAUNCH_CHECK("depth_filter_kernel");
  return HS2_OK;
}
