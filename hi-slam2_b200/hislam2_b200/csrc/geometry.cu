// iproj / covis_distance / depth_filter: the per-pixel back-projection helpers of the
// keyframe policy and of the point-cloud filter (reference: src/droid_kernels.cu
// covis_distance_kernel :996-1090, depth_filter_kernel :1094-1204, iproj_kernel
// :1208-1272, host wrappers :2071-2143); proj_trans / bi_inter: the two operators of the
// mono-depth-prior alignment (JDSA, hislam2/geom/ba.py:161-219; reference
// projective_transform2_kernel :246-362 + proj_trans_cuda :1781-1818, bi_inter_kernel
// :1275-1316 + bi_inter_cuda :2145-2175).
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
//   proj_trans      CTA per edge: the depth-only Schur terms C = wu Jzu^2 + wv Jzv^2 and
//                   w = wu ru Jzu + wv rv Jzv of every pixel (the ba linearisation without
//                   the pose blocks), added with atomics into the row slot[e] of the edge's
//                   source frame (the reference's accum_cuda over kx = unique(ii)).
//   bi_inter        thread per pixel: bilinear interpolation of the frame's scale grid at
//                   (x, y) and the four non-zero entries of the dense Jacobian
//                   [N,H,W,hs,ws] (zeroed first), as the reference writes them.
// Entries whose frame index lies outside the buffers (the reference reads out of bounds
// there) set HS2_DEV_BAD_INDEX and produce no output for that entry.
#include <algorithm>

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

__global__ void __launch_bounds__(kGeoThreads)
proj_trans_kernel(const float* __restrict__ poses, int64_t num_poses, const float* __restrict__ disps,
                  int64_t num_disps, int ht, int wd, const float* __restrict__ intr,
                  const float* __restrict__ targets, const float* __restrict__ weights,
                  const int64_t* __restrict__ ii, const int64_t* __restrict__ jj, const int64_t* __restrict__ slot,
                  int64_t num_slots, float* __restrict__ C, float* __restrict__ w, int32_t* __restrict__ info) {
  const int e = blockIdx.x;
  const int64_t ix = ii[e], jx = jj[e], m = slot[e];
  if (ix < 0 || jx < 0 || ix >= num_poses || jx >= num_poses || ix >= num_disps || m < 0 || m >= num_slots) {
    if (threadIdx.x == 0) atomicOr(info, HS2_DEV_BAD_INDEX);
    return;
  }
  const float fx = intr[0], fy = intr[1], cx = intr[2], cy = intr[3];
  float tij[3], qij[4];
  relative_pose(poses + 7 * ix, poses + 7 * ix + 3, poses + 7 * jx, poses + 7 * jx + 3, tij, qij);
  const int HW = ht * wd;
  const float* drow = disps + ix * HW;
  const float* trg = targets + (int64_t)e * 2 * HW;
  const float* wgt = weights + (int64_t)e * 2 * HW;
  float* Cm = C + m * HW;
  float* wm = w + m * HW;
  for (int k = blockIdx.y * kGeoThreads + threadIdx.x; k < HW; k += gridDim.y * kGeoThreads) {
    const int vi = k / wd;
    const float u = (float)(k - vi * wd), v = (float)vi;
    const float X[3] = {(u - cx) / fx, (v - cy) / fy, 1.0f};
    const float h = drow[k];
    float Y[3];
    quat_rotate(qij, X, Y);
    Y[0] += h * tij[0]; Y[1] += h * tij[1]; Y[2] += h * tij[2];
    const bool bad = Y[2] < kMinDepth;
    const float xp = fx * (Y[0] / Y[2]) + cx, yp = fy * (Y[1] / Y[2]) + cy;
    const float d = bad ? 0.f : 1.0f / Y[2];
    const float d2 = d * d;
    const float wu = bad ? 0.f : 0.001f * wgt[k];
    const float wv = bad ? 0.f : 0.001f * wgt[HW + k];
    const float ru = trg[k] - xp, rv = trg[HW + k] - yp;
    const float Jzu = fx * d * tij[0] + fx * (-Y[0] * d2) * tij[2];
    const float Jzv = fy * d * tij[1] + fy * (-Y[1] * d2) * tij[2];
    atomicAdd(&Cm[k], wu * Jzu * Jzu + wv * Jzv * Jzv);
    atomicAdd(&wm[k], wu * ru * Jzu + wv * rv * Jzv);
  }
}

__global__ void __launch_bounds__(kGeoThreads)
bi_inter_kernel(const float* __restrict__ scales, int hs, int ws, const float* __restrict__ grids, int ht, int wd,
                float* __restrict__ out, float* __restrict__ jac, int32_t* __restrict__ info) {
  const int b = blockIdx.y;
  const int HW = ht * wd;
  const int k = blockIdx.x * kGeoThreads + threadIdx.x;
  if (k >= HW) return;
  const float x = grids[((int64_t)b * HW + k) * 2 + 0];
  const float y = grids[((int64_t)b * HW + k) * 2 + 1];
  const int x0 = (int)floorf(x), y0 = (int)floorf(y);
  const int x1 = x0 + 1, y1 = y0 + 1;
  if (!(x0 >= 0 && y0 >= 0 && x1 < ws && y1 < hs)) {   // also false for NaN
    out[(int64_t)b * HW + k] = 0.f;
    atomicOr(info, HS2_DEV_BAD_INDEX);
    return;
  }
  const float wa = ((float)x1 - x) * ((float)y1 - y), wb = ((float)x1 - x) * (y - (float)y0);
  const float wc = (x - (float)x0) * ((float)y1 - y), wdd = (x - (float)x0) * (y - (float)y0);
  const float* S = scales + (int64_t)b * hs * ws;
  out[(int64_t)b * HW + k] = wa * S[y0 * ws + x0] + wb * S[y1 * ws + x0] + wc * S[y0 * ws + x1] + wdd * S[y1 * ws + x1];
  float* J = jac + ((int64_t)b * HW + k) * hs * ws;
  J[y0 * ws + x0] = wa;
  J[y1 * ws + x0] = wb;
  J[y0 * ws + x1] = wc;
  J[y1 * ws + x1] = wdd;
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

extern "C" int hs2_proj_trans(const float* poses, int64_t num_poses, const float* disps, int64_t num_disps, int ht,
                              int wd, const float* intrinsics, const float* targets, const float* weights,
                              const int64_t* ii, const int64_t* jj, const int64_t* slot, int64_t num_edges,
                              int64_t num_slots, float* C, float* w, int32_t* info, hs2_stream_t stream) {
  using namespace hs2;
  int rc = check_geo("proj_trans", num_poses, num_disps, ht, wd);
  if (rc) return rc;
  if (num_edges < 0 || num_edges > 0x7fffffff || num_slots < 0) {
    set_error("proj_trans: bad counts (edges %lld, slots %lld)", (long long)num_edges, (long long)num_slots);
    return HS2_ERR_INVALID;
  }
  if (num_slots == 0) return HS2_OK;
  if ((rc = bind_device(C))) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  const int HW = ht * wd;
  HS2_CUDA(cudaMemsetAsync(C, 0, sizeof(float) * (size_t)num_slots * HW, s));
  HS2_CUDA(cudaMemsetAsync(w, 0, sizeof(float) * (size_t)num_slots * HW, s));
  if (num_edges == 0) return HS2_OK;
  const int ysplit = std::min(8, (HW + kGeoThreads - 1) / kGeoThreads);
  HS2_PROF("proj_trans", s);
  proj_trans_kernel<<<dim3((unsigned)num_edges, ysplit), kGeoThreads, 0, s>>>(
      poses, num_poses, disps, num_disps, ht, wd, intrinsics, targets, weights, ii, jj, slot, num_slots, C, w, info);
  HS2_LAUNCH_CHECK("proj_trans_kernel");
  return HS2_OK;
}

extern "C" int hs2_bi_inter(const float* scales, int64_t num, int hs, int ws, const float* grids, int ht, int wd,
                            float* outputs, float* jacobians, int32_t* info, hs2_stream_t stream) {
  using namespace hs2;
  if (num < 0 || num > 65535 || hs <= 0 || ws <= 0 || ht <= 0 || wd <= 0 || (int64_t)ht * wd > (1 << 30)) {
    set_error("bi_inter: bad sizes num=%lld hs=%d ws=%d ht=%d wd=%d", (long long)num, hs, ws, ht, wd);
    return HS2_ERR_INVALID;
  }
  if (num == 0) return HS2_OK;
  int rc = bind_device(outputs);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  const int HW = ht * wd;
  HS2_CUDA(cudaMemsetAsync(jacobians, 0, sizeof(float) * (size_t)num * HW * hs * ws, s));
  HS2_PROF("bi_inter", s);
  bi_inter_kernel<<<dim3((HW + kGeoThreads - 1) / kGeoThreads, (unsigned)num), kGeoThreads, 0, s>>>(
      scales, hs, ws, grids, ht, wd, outputs, jacobians, info);
  HS2_LAUNCH_CHECK("bi_inter_kernel");
  return HS2_OK;
}
