// frame_distance: per-edge mean optical-flow magnitude used for keyframe
// selection (reference: src/droid_kernels.cu:860-994, host side :2047-2069).
//
// One CTA per edge; each thread walks a strided set of pixels, the three sums
// are reduced with warp shuffles and one shared-memory pass.  HBM traffic is one
// disparity row per edge (4*ht*wd bytes).
#include "common.cuh"
#include "profile.cuh"

namespace hs2 {

constexpr int kFdThreads = 256;

__global__ void __launch_bounds__(kFdThreads)
frame_distance_kernel(const float* __restrict__ poses, int64_t num_poses,
                      const float* __restrict__ disps, int64_t num_disps, int ht, int wd,
                      const float* __restrict__ intr, const int64_t* __restrict__ ii,
                      const int64_t* __restrict__ jj, float beta, float* __restrict__ dist,
                      int32_t* __restrict__ info) {
  const int e = blockIdx.x;
  const int64_t ix = ii[e], jx = jj[e];
  if (ix < 0 || jx < 0 || ix >= num_poses || jx >= num_poses || ix >= num_disps) {
    if (threadIdx.x == 0) {
      dist[e] = 1000.0f;
      if (info) atomicOr(info, HS2_DEV_BAD_INDEX);
    }
    return;
  }
  const float fx = intr[0], fy = intr[1], cx = intr[2], cy = intr[3];
  float tij[3], qij[4];
  relative_pose(poses + 7 * ix, poses + 7 * ix + 3, poses + 7 * jx, poses + 7 * jx + 3, tij, qij);

  const int HW = ht * wd;
  const float* d_row = disps + (int64_t)ix * HW;
  const float nbeta = 1.0f - beta;
  float acc = 0.f, val = 0.f, tot = 0.f;
  for (int k = threadIdx.x; k < HW; k += kFdThreads) {
    const float v = (float)(k / wd);
    const float u = (float)(k - (k / wd) * wd);
    const float X[3] = {(u - cx) / fx, (v - cy) / fy, 1.0f};
    const float d = d_row[k];
    float Y[3];
    quat_rotate(qij, X, Y);
    Y[0] += d * tij[0]; Y[1] += d * tij[1]; Y[2] += d * tij[2];
    float du = fx * (Y[0] / Y[2]) + cx - u;
    float dv = fy * (Y[1] / Y[2]) + cy - v;
    tot += beta;
    if (Y[2] > kMinDepth) {
      acc += beta * sqrtf(du * du + dv * dv);
      val += beta;
    }
    // translation only
    const float Z[3] = {X[0] + d * tij[0], X[1] + d * tij[1], X[2] + d * tij[2]};
    du = fx * (Z[0] / Z[2]) + cx - u;
    dv = fy * (Z[1] / Z[2]) + cy - v;
    tot += nbeta;
    if (Z[2] > kMinDepth) {
      acc += nbeta * sqrtf(du * du + dv * dv);
      val += nbeta;
    }
  }
  acc = warp_sum(acc);
  val = warp_sum(val);
  tot = warp_sum(tot);
  __shared__ float red[3][kFdThreads / 32];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) { red[0][wid] = acc; red[1][wid] = val; red[2][wid] = tot; }
  __syncthreads();
  if (wid == 0) {
    acc = lane < kFdThreads / 32 ? red[0][lane] : 0.f;
    val = lane < kFdThreads / 32 ? red[1][lane] : 0.f;
    tot = lane < kFdThreads / 32 ? red[2][lane] : 0.f;
    acc = warp_sum(acc);
    val = warp_sum(val);
    tot = warp_sum(tot);
    if (lane == 0) dist[e] = (val / (tot + 1e-8f) < 0.75f) ? 1000.0f : acc / val;
  }
}

}  // namespace hs2

extern "C" int hs2_frame_distance(const float* poses, int64_t num_poses, const float* disps,
                                  int64_t num_disps, int ht, int wd, const float* intrinsics,
                                  const int64_t* ii, const int64_t* jj, int64_t num_edges, float beta,
                                  float* dist, int32_t* info, hs2_stream_t stream) {
  using namespace hs2;
  if (num_edges < 0 || ht <= 0 || wd <= 0 || num_poses < 0 || num_disps < 0) {
    set_error("frame_distance: bad sizes (edges=%lld ht=%d wd=%d)", (long long)num_edges, ht, wd);
    return HS2_ERR_INVALID;
  }
  if (num_edges == 0) return HS2_OK;
  if (num_edges > 0x7fffffff) {
    set_error("frame_distance: too many edges");
    return HS2_ERR_INVALID;
  }
  int rc = bind_device(dist);
  if (rc) return rc;
  HS2_PROF("frame_distance", (cudaStream_t)stream);
  frame_distance_kernel<<<(unsigned)num_edges, kFdThreads, 0, (cudaStream_t)stream>>>(
      poses, num_poses, disps, num_disps, ht, wd, intrinsics, ii, jj, beta, dist, info);
  HS2_LAUNCH_CHECK("frame_distance_kernel");
  return HS2_OK;
}
