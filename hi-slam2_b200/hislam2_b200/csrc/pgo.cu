// Pose-graph terms around pgba: the relative Sim3 pose factors' blocks Hsp / vsp
// (HI-SLAM2 hislam2/pgo_buffer.py:39-63, global_relative_posesim3_constraints) and the
// Sim3 retraction of the window after each pgba step (hislam2/depth_video.py:267,
// geom/ba.py:27-29 pose_retr with lietorch's Sim3.retr).  The reference evaluates the
// factors with lietorch on [1, Np] batches: 28 exp / mul / inv / log passes for the
// central-difference Jacobians, then a dozen float32 matmuls; here one launch does it all.
//
//   pgo_constraints  CTA of 8 factors x 16 lanes.  Lanes 0..13 each form one Jacobian
//                    column (a +-1e-8 pair of perturbed log(Gij Gi Gj^-1), FP64), lane 14
//                    the residual; the table (rounded to float) goes to shared memory;
//                    then the lanes share the factor's 98 wJ^T entries (FP64 sums of the
//                    float Jacobians times the information, rounded), and its 4 x 49 Hsp,
//                    2 x 7 vsp and 2 chi^2 terms.  Factors whose pose index is outside
//                    the buffer get zero blocks and set HS2_DEV_BAD_INDEX.
//   sim3_retr        thread per pose of [t0, t1): G <- exp(dx) G in FP64, stored as float.
#include "common.cuh"
#include "profile.cuh"
#include "sim3.cuh"

namespace hs2 {

namespace {

constexpr int kPgoFactors = 8;
constexpr int kPgoLanes = 16;
constexpr int kPgoThreads = kPgoFactors * kPgoLanes;
constexpr int kPgoOut = 4 * 49 + 2 * 7 + 2;   // Hsp, vsp and chi^2 entries of one factor

__global__ void __launch_bounds__(kPgoThreads)
pgo_constraints_kernel(const float* __restrict__ poses, int64_t num_poses, const int64_t* __restrict__ ii,
                       const int64_t* __restrict__ jj, const float* __restrict__ rel, const float* __restrict__ infos,
                       int64_t num_factors, double pw, float* __restrict__ Hsp, float* __restrict__ vsp,
                       float* __restrict__ chi, int32_t* __restrict__ info) {
  __shared__ float J[kPgoFactors][15][8];
  __shared__ float W[kPgoFactors][2][7][8];
  const int f = threadIdx.x / kPgoLanes, lane = threadIdx.x % kPgoLanes;
  const int64_t n = (int64_t)blockIdx.x * kPgoFactors + f;
  bool ok = n < num_factors;
  int64_t i = 0, j = 0;
  if (ok) {
    i = ii[n];
    j = jj[n];
    if (i < 0 || j < 0 || i >= num_poses || j >= num_poses) {
      ok = false;
      if (lane == 0) atomicOr(info, HS2_DEV_BAD_INDEX);
    }
  }
  if (ok && lane < 15) {
    const sim3::Sim3d Gi = sim3::from_floats(poses + 8 * i, true);
    const sim3::Sim3d Gj = sim3::from_floats(poses + 8 * j, true);
    const sim3::Sim3d Gij = sim3::from_floats(rel + 7 * n, false);
    double col[7];
    sim3::factor_column(Gi, Gj, Gij, lane, col);
#pragma unroll
    for (int a = 0; a < 7; ++a) J[f][lane][a] = (float)col[a];
  }
  __syncthreads();
  const float* inf = infos + 49 * (ok ? n : 0);
  if (ok) {
    for (int e = lane; e < 98; e += kPgoLanes) {
      const int x = e / 49, a = (e % 49) / 7, b = e % 7;
      W[f][x][a][b] = sim3::wjt_entry(J[f], inf, x, a, b, pw);
    }
  }
  __syncthreads();
  if (n >= num_factors) return;
  for (int e = lane; e < kPgoOut; e += kPgoLanes) {
    if (e < 196) {
      const int blk = e / 49, a = (e % 49) / 7, b = e % 7;
      Hsp[((int64_t)blk * num_factors + n) * 49 + a * 7 + b] = ok ? sim3::hsp_entry(W[f], J[f], blk, a, b) : 0.f;
    } else if (e < 210) {
      const int x = (e - 196) / 7, a = (e - 196) % 7;
      vsp[((int64_t)x * num_factors + n) * 7 + a] = ok ? sim3::vsp_entry(W[f], J[f], x, a) : 0.f;
    } else {
      const int sc = e - 210;
      chi[2 * n + sc] = ok ? sim3::chi_entry(J[f], inf, sc) : 0.f;
    }
  }
}

__global__ void __launch_bounds__(128)
sim3_retr_kernel(float* __restrict__ poses, const float* __restrict__ dx, int64_t t0, int64_t count) {
  const int64_t k = (int64_t)blockIdx.x * 128 + threadIdx.x;
  if (k >= count) return;
  float* p = poses + 8 * (t0 + k);
  double xi[7];
#pragma unroll
  for (int a = 0; a < 7; ++a) xi[a] = (double)dx[7 * k + a];
  const sim3::Sim3d G = sim3::mul(sim3::exp(xi), sim3::from_floats(p, true));
#pragma unroll
  for (int a = 0; a < 3; ++a) p[a] = (float)G.t[a];
#pragma unroll
  for (int a = 0; a < 4; ++a) p[3 + a] = (float)G.q[a];
  p[7] = (float)G.s;
}

}  // namespace
}  // namespace hs2

extern "C" int hs2_pgo_constraints(const float* poses, int64_t num_poses, const int64_t* ii, const int64_t* jj,
                                   const float* rel_poses, const float* infos, int64_t num_factors, double pw,
                                   float* Hsp, float* vsp, float* chi, int32_t* info, hs2_stream_t stream) {
  using namespace hs2;
  if (num_poses < 0 || num_factors < 0 || num_factors > ((int64_t)1 << 31) * kPgoFactors / 2) {
    set_error("pgo_constraints: bad sizes (poses %lld, factors %lld)", (long long)num_poses,
              (long long)num_factors);
    return HS2_ERR_INVALID;
  }
  if (!info) {
    set_error("pgo_constraints: info is null");
    return HS2_ERR_INVALID;
  }
  int rc = bind_device(info);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  HS2_CUDA(cudaMemsetAsync(info, 0, sizeof(int32_t), s));
  if (num_factors == 0) return HS2_OK;
  HS2_PROF("pgo_constraints", s);
  pgo_constraints_kernel<<<(unsigned)((num_factors + kPgoFactors - 1) / kPgoFactors), kPgoThreads, 0, s>>>(
      poses, num_poses, ii, jj, rel_poses, infos, num_factors, pw, Hsp, vsp, chi, info);
  HS2_LAUNCH_CHECK("pgo_constraints_kernel");
  return HS2_OK;
}

extern "C" int hs2_sim3_retr(float* poses, int64_t num_poses, const float* dx, int64_t t0, int64_t t1,
                             hs2_stream_t stream) {
  using namespace hs2;
  if (t0 < 0 || t1 < t0 || t1 > num_poses || t1 - t0 > ((int64_t)1 << 31)) {
    set_error("sim3_retr: window [%lld, %lld) outside %lld poses", (long long)t0, (long long)t1,
              (long long)num_poses);
    return HS2_ERR_INVALID;
  }
  if (t1 == t0) return HS2_OK;
  int rc = bind_device(poses);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  HS2_PROF("sim3_retr", s);
  sim3_retr_kernel<<<(unsigned)((t1 - t0 + 127) / 128), 128, 0, s>>>(poses, dx, t0, t1 - t0);
  HS2_LAUNCH_CHECK("sim3_retr_kernel");
  return HS2_OK;
}
