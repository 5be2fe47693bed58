// Reprojection + multi-level correlation lookup in one launch (the caller side of
// HI-SLAM2's update step fused):
//   coords1 = DepthVideo.reproject(ii, jj)        hislam2/depth_video.py:170-178
//   corr    = AltCorrBlock(fmaps)(coords1, ii, jj) hislam2/modules/corr.py:90-117
// (factor_graph.py:194-200, :253-260).  Per (edge, level, 32 pixels) a CTA projects
// its pixels of frame ii into frame jj with Gij = Gj Gi^-1 (float, as the reference's
// lietorch projective_transform), scales the coordinates by 2^-level, and forms the
// (2r+1)^2 bilinear window of correlations against the level's pooled features of
// frame jj on the fly, as altcorr_forward does.  Neither the coordinates (except an
// optional level-0 copy for the motion features) nor any correlation volume is
// written to memory.  Output layout [E, levels * (2r+1)^2, H, W]: the concatenation
// over levels that AltCorrBlock / CorrBlock.__call__ return (dim 2 ordered level,
// then x offset, then y offset).
#include "common.cuh"
#include "profile.cuh"

namespace hs2 {

constexpr int kCfThreads = 256;
constexpr int kCfPix = 32;
constexpr int kCfTaps = 16;

struct CfLevels {
  const void* f[4];        // pooled features of every frame, level l: [K, C, H >> l, W >> l]
};

template <typename T>
__global__ void __launch_bounds__(kCfThreads)
corr_fused_kernel(const float* __restrict__ poses, int64_t num_poses, const float* __restrict__ disps,
                  int64_t num_disps, const float* __restrict__ intr, CfLevels lv, int64_t K, int C, int H, int W,
                  const int64_t* __restrict__ ii, const int64_t* __restrict__ jj, int levels, int r, int stride,
                  T* __restrict__ corr, float* __restrict__ coords_out, int32_t* __restrict__ info) {
  extern __shared__ float4 cf_smem[];
  float4* geo = cf_smem;
  float* win = reinterpret_cast<float*>(cf_smem) + 4 * kCfPix;
  __shared__ float G[12];                       // R (row-major) then t of Gij

  const int m = blockIdx.y, lvl = blockIdx.z;
  const int HW = H * W;
  const int H2 = H >> lvl, W2 = W >> lvl;
  const int64_t HW2 = (int64_t)H2 * W2;
  const int pix0 = blockIdx.x * kCfPix;
  const int D = 2 * r + 2, rd = 2 * r + 1;
  const int64_t ix = ii[m], jx = jj[m];
  const bool ok = ix >= 0 && jx >= 0 && ix < K && jx < K && ix < num_poses && jx < num_poses && ix < num_disps;
  if (!ok && threadIdx.x == 0 && blockIdx.x == 0 && lvl == 0) atomicOr(info, HS2_DEV_BAD_INDEX);
  if (threadIdx.x == 0) {
    float t[3], q[4];
    if (ok) {
      relative_pose(poses + 7 * ix, poses + 7 * ix + 3, poses + 7 * jx, poses + 7 * jx + 3, t, q);
    } else {
      t[0] = t[1] = t[2] = 0.f;
      q[0] = q[1] = q[2] = 0.f;
      q[3] = 1.f;
    }
    const float x = q[0], y = q[1], z = q[2], w = q[3];
    G[0] = 1.f - 2.f * (y * y + z * z); G[1] = 2.f * (x * y - z * w);       G[2] = 2.f * (x * z + y * w);
    G[3] = 2.f * (x * y + z * w);       G[4] = 1.f - 2.f * (x * x + z * z); G[5] = 2.f * (y * z - x * w);
    G[6] = 2.f * (x * z - y * w);       G[7] = 2.f * (y * z + x * w);       G[8] = 1.f - 2.f * (x * x + y * y);
    G[9] = t[0]; G[10] = t[1]; G[11] = t[2];
  }
  __syncthreads();
  const float fx = intr[0], fy = intr[1], cx = intr[2], cy = intr[3];
  const float scale = 1.0f / (float)(1 << lvl);
  for (int q = threadIdx.x; q < kCfPix; q += kCfThreads) {
    const int pix = min(pix0 + q, HW - 1);
    const int v = pix / W, u = pix - v * W;
    const float d = ok ? disps[ix * HW + pix] : 0.f;
    const float X = (u - cx) / fx, Y = (v - cy) / fy;
    const float P0 = G[0] * X + G[1] * Y + G[2] + G[9] * d;
    const float P1 = G[3] * X + G[4] * Y + G[5] + G[10] * d;
    const float P2 = G[6] * X + G[7] * Y + G[8] + G[11] * d;
    const float xc = fx * (P0 / P2) + cx, yc = fy * (P1 / P2) + cy;
    if (lvl == 0 && coords_out && pix0 + q < HW) {
      coords_out[((int64_t)m * HW + pix) * 2 + 0] = xc;
      coords_out[((int64_t)m * HW + pix) * 2 + 1] = yc;
    }
    const float xs = xc * scale, ys = yc * scale;
    const float flx = floorf(xs), fly = floorf(ys);
    geo[q] = make_float4(xs - flx, ys - fly, __int_as_float((int)flx - r), __int_as_float((int)fly - r));
  }
  __syncthreads();

  const T* f1 = static_cast<const T*>(lv.f[0]) + (ok ? ix : 0) * C * (int64_t)HW;
  const T* f2 = static_cast<const T*>(lv.f[lvl]) + (ok ? jx : 0) * C * HW2;
  for (int item = threadIdx.x; item < kCfPix * D; item += kCfThreads) {
    const int py = item / kCfPix;
    const int q = item - py * kCfPix;
    const int pix = pix0 + q;
    float* wrow = win + q * stride + py * D;
    const float4 g = geo[q];
    const int y1 = __float_as_int(g.w) + py;
    const int xb = __float_as_int(g.z);
    const bool row_ok = ok && pix < HW && y1 >= 0 && y1 < H2;
    for (int c0 = 0; c0 < D; c0 += kCfTaps) {
      float acc[kCfTaps];
#pragma unroll
      for (int k = 0; k < kCfTaps; ++k) acc[k] = 0.f;
      if (row_ok) {
        const T* a = f1 + pix;
        const T* brow = f2 + (int64_t)y1 * W2;
        for (int c = 0; c < C; ++c) {
          const float av = to_f(a[(int64_t)c * HW]);
          const T* bc = brow + (int64_t)c * HW2;
#pragma unroll
          for (int k = 0; k < kCfTaps; ++k) {
            const int x1 = xb + c0 + k;
            if (c0 + k < D && x1 >= 0 && x1 < W2) acc[k] += av * to_f(bc[x1]);
          }
        }
      }
#pragma unroll
      for (int k = 0; k < kCfTaps; ++k)
        if (c0 + k < D) wrow[c0 + k] = acc[k] * 0.0625f;
    }
  }
  __syncthreads();

  const int nout = rd * rd;
  T* out = corr + ((int64_t)m * levels + lvl) * nout * HW;
  for (int idx = threadIdx.x; idx < kCfPix * nout; idx += kCfThreads) {
    const int o = idx / kCfPix;
    const int q = idx - o * kCfPix;
    const int pix = pix0 + q;
    if (pix >= HW) continue;
    const int a = o / rd, bb = o - a * rd;
    const float4 g = geo[q];
    const float* w = win + q * stride;
    const float v = (1.f - g.x) * (1.f - g.y) * w[bb * D + a] + g.x * (1.f - g.y) * w[bb * D + a + 1] +
                    (1.f - g.x) * g.y * w[(bb + 1) * D + a] + g.x * g.y * w[(bb + 1) * D + a + 1];
    out[(int64_t)o * HW + pix] = from_f<T>(v);
  }
}

template <typename T>
static int cf_launch(const float* poses, int64_t np, const float* disps, int64_t nd, const float* intr,
                     CfLevels lv, int64_t K, int C, int H, int W, const int64_t* ii, const int64_t* jj, int64_t E,
                     int levels, int r, void* corr, float* coords_out, int32_t* info, cudaStream_t s) {
  const int D = 2 * r + 2;
  int stride = D * D;
  if ((stride & 1) == 0) stride += 1;
  const size_t smem = (size_t)kCfPix * (stride * 4 + 16);
  if (smem > 48 * 1024)
    HS2_CUDA(cudaFuncSetAttribute(corr_fused_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  dim3 grid((H * W + kCfPix - 1) / kCfPix, (unsigned)E, levels);
  HS2_PROF("corr_fused", s);
  corr_fused_kernel<T><<<grid, kCfThreads, smem, s>>>(poses, np, disps, nd, intr, lv, K, C, H, W, ii, jj, levels, r,
                                                      stride, static_cast<T*>(corr), coords_out, info);
  HS2_LAUNCH_CHECK("corr_fused_kernel");
  return HS2_OK;
}

}  // namespace hs2

extern "C" int hs2_corr_reproject_lookup(const float* poses, int64_t num_poses, const float* disps,
                                         int64_t num_disps, const float* intrinsics, const void* const* fmap_levels,
                                         int levels, int dtype, int64_t num_frames, int channels, int ht, int wd,
                                         const int64_t* ii, const int64_t* jj, int64_t num_edges, int radius,
                                         void* corr, float* coords1, int32_t* info, hs2_stream_t stream) {
  using namespace hs2;
  if (levels < 1 || levels > 4 || radius < 0 || radius > 30 || channels <= 0 || ht <= 0 || wd <= 0 ||
      num_edges < 0 || num_edges > 65535 || num_frames <= 0 || (ht >> (levels - 1)) <= 0 ||
      (wd >> (levels - 1)) <= 0) {
    set_error("corr_reproject_lookup: bad sizes (levels=%d r=%d C=%d ht=%d wd=%d E=%lld K=%lld)", levels, radius,
              channels, ht, wd, (long long)num_edges, (long long)num_frames);
    return HS2_ERR_INVALID;
  }
  if (num_edges == 0) return HS2_OK;
  if (!poses || !disps || !intrinsics || !fmap_levels || !ii || !jj || !corr || !info) {
    set_error("corr_reproject_lookup: null pointer argument");
    return HS2_ERR_INVALID;
  }
  CfLevels lv;
  for (int l = 0; l < 4; ++l) lv.f[l] = l < levels ? fmap_levels[l] : nullptr;
  for (int l = 0; l < levels; ++l)
    if (!lv.f[l]) {
      set_error("corr_reproject_lookup: feature level %d missing", l);
      return HS2_ERR_INVALID;
    }
  int rc;
  if ((rc = bind_device(corr))) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  switch (dtype) {
    case HS2_F32:
      return cf_launch<float>(poses, num_poses, disps, num_disps, intrinsics, lv, num_frames, channels, ht, wd, ii, jj,
                              num_edges, levels, radius, corr, coords1, info, s);
    case HS2_F16:
      return cf_launch<__half>(poses, num_poses, disps, num_disps, intrinsics, lv, num_frames, channels, ht, wd, ii,
                               jj, num_edges, levels, radius, corr, coords1, info, s);
    case HS2_BF16:
      return cf_launch<__nv_bfloat16>(poses, num_poses, disps, num_disps, intrinsics, lv, num_frames, channels, ht,
                                      wd, ii, jj, num_edges, levels, radius, corr, coords1, info, s);
  }
  set_error("corr_reproject_lookup: unsupported dtype %d (f32, f16, bf16)", dtype);
  return HS2_ERR_DTYPE;
}
