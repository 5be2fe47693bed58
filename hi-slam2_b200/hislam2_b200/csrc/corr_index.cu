// corr_index_forward / corr_index_backward: radius-r bilinear lookup into a
// precomputed all-pairs correlation volume and its adjoint
// (reference: src/correlation_kernels.cu:19-184).
//
// Layout: volume [n, h1, w1, h2, w2] (one h2*w2 plane per source pixel),
// coords [n, 2, h1, w1] (x then y), corr [n, 2r+1, 2r+1, h1, w1] with dim 1 along x.
//
// Forward: a CTA owns `tpix` consecutive source pixels of one image.  Phase 1
// stages each pixel's (2r+2)^2 window in shared memory with lanes running along
// the window rows (contiguous in x1), phase 2 forms the (2r+1)^2 bilinear
// outputs with consecutive threads on consecutive pixels, so every store of a
// warp is one contiguous segment.  The op is a gather: HBM-bound on the window
// reads.
//
// Backward: the same CTA tiling; each CTA writes its pixels' whole h2*w2 planes
// of volume_grad (zeros with 16-byte stores, then the window values), i.e. one
// streaming write of the volume instead of a memset followed by a scatter.
#include "common.cuh"
#include "profile.cuh"

namespace hs2 {

constexpr int kCiThreads = 256;

struct CiTile {
  int tpix;     // source pixels per CTA
  int D;        // window side 2r+2
  int stride;   // floats per pixel window in smem (D*D padded to odd)
  size_t smem;  // dynamic smem bytes
};

static CiTile ci_tile(int radius, int out_side) {
  CiTile t;
  t.D = 2 * radius + 2;
  t.stride = t.D * t.D;
  if ((t.stride & 1) == 0) t.stride += 1;
  (void)out_side;
  const size_t per_pix = (size_t)t.stride * 4 + 16;
  int tp = (int)((96 * 1024) / per_pix);
  if (tp > 64) tp = 64;
  if (tp < 1) tp = 1;
  t.tpix = tp;
  t.smem = (size_t)tp * per_pix;
  return t;
}

template <typename T>
__global__ void __launch_bounds__(kCiThreads)
corr_index_fwd_kernel(const T* __restrict__ volume, const float* __restrict__ coords, T* __restrict__ corr,
                      int h1, int w1, int h2, int w2, int r, int tpix, int stride) {
  extern __shared__ float4 smem4[];
  float2* frac = reinterpret_cast<float2*>(smem4);                  // [tpix] fractional coords
  float* win = reinterpret_cast<float*>(smem4) + 4 * (size_t)tpix;  // [tpix][stride]

  const int n = blockIdx.y;
  const int HW1 = h1 * w1;
  const int64_t HW2 = (int64_t)h2 * w2;
  const int pix0 = blockIdx.x * tpix;
  const int D = 2 * r + 2;
  const int rd = 2 * r + 1;
  const int DD = D * D;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int nwarp = kCiThreads / 32;

  // phase 1: windows
  for (int p = warp; p < tpix; p += nwarp) {
    const int pix = pix0 + p;
    if (pix >= HW1) break;
    const float cx = coords[((int64_t)n * 2 + 0) * HW1 + pix];
    const float cy = coords[((int64_t)n * 2 + 1) * HW1 + pix];
    const float fx = floorf(cx), fy = floorf(cy);
    const int x0 = (int)fx - r, y0 = (int)fy - r;
    if (lane == 0) frac[p] = make_float2(cx - fx, cy - fy);
    const T* plane = volume + ((int64_t)n * HW1 + pix) * HW2;
    for (int t = lane; t < DD; t += 32) {
      const int jy = t / D;
      const int ix = t - jy * D;
      const int x1 = x0 + ix, y1 = y0 + jy;
      float v = 0.f;
      if (x1 >= 0 && x1 < w2 && y1 >= 0 && y1 < h2) v = to_f(plane[(int64_t)y1 * w2 + x1]);
      win[p * stride + t] = v;
    }
  }
  __syncthreads();

  // phase 2: bilinear outputs, consecutive threads -> consecutive pixels
  const int nout = rd * rd;
  for (int idx = threadIdx.x; idx < tpix * nout; idx += kCiThreads) {
    const int o = idx / tpix;
    const int p = idx - o * tpix;
    const int pix = pix0 + p;
    if (pix >= HW1) continue;
    const int a = o / rd;       // x offset
    const int b = o - a * rd;   // y offset
    const float2 f = frac[p];
    const float* w = win + p * stride;
    const float v00 = w[b * D + a], v01 = w[(b + 1) * D + a];
    const float v10 = w[b * D + a + 1], v11 = w[(b + 1) * D + a + 1];
    const float val = (1.f - f.x) * (1.f - f.y) * v00 + (1.f - f.x) * f.y * v01 +
                      f.x * (1.f - f.y) * v10 + f.x * f.y * v11;
    corr[((int64_t)n * nout + o) * HW1 + pix] = from_f<T>(val);
  }
}

// Forward for a compile-time radius (the network's r = 3 and the r = 4 of the lookup
// benchmarks): 64 source pixels per CTA; their window origins and fractions are
// staged first, then every warp gathers the (2R+2)^2 windows of 8 pixels with all its
// loads issued back to back (tap index -> (row, column) by constant division), and
// the (2R+1)^2 outputs are formed four threads per pixel, stores contiguous along
// the pixels.
template <typename T, int R>
__global__ void __launch_bounds__(kCiThreads)
corr_index_fwd_r_kernel(const T* __restrict__ volume, const float* __restrict__ coords, T* __restrict__ corr,
                        int h1, int w1, int h2, int w2) {
  constexpr int D = 2 * R + 2, DD = D * D, RD = 2 * R + 1, NOUT = RD * RD;
  constexpr int TP = 64, STRIDE = (DD & 1) ? DD : DD + 1;
  constexpr int NT = (DD + 31) / 32;
  __shared__ float win[TP * STRIDE];
  __shared__ float2 frac[TP];
  __shared__ int2 org[TP];
  const int n = blockIdx.y;
  const int HW1 = h1 * w1;
  const int64_t HW2 = (int64_t)h2 * w2;
  const int pix0 = blockIdx.x * TP;
  if (threadIdx.x < TP) {
    const int pix = min(pix0 + (int)threadIdx.x, HW1 - 1);
    const float cx = coords[((int64_t)n * 2 + 0) * HW1 + pix];
    const float cy = coords[((int64_t)n * 2 + 1) * HW1 + pix];
    const float fx = floorf(cx), fy = floorf(cy);
    frac[threadIdx.x] = make_float2(cx - fx, cy - fy);
    org[threadIdx.x] = make_int2((int)fx - R, (int)fy - R);
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll 2
  for (int q = 0; q < TP / 8; ++q) {
    const int p = warp * (TP / 8) + q;
    const int pix = min(pix0 + p, HW1 - 1);
    const int2 o = org[p];
    const T* plane = volume + ((int64_t)n * HW1 + pix) * HW2;
    float v[NT];
#pragma unroll
    for (int k = 0; k < NT; ++k) {
      const int t = lane + 32 * k;
      const int jy = t / D, ix = t - (t / D) * D;
      const int x1 = o.x + ix, y1 = o.y + jy;
      v[k] = 0.f;
      if (t < DD && x1 >= 0 && x1 < w2 && y1 >= 0 && y1 < h2) v[k] = to_f(plane[(int64_t)y1 * w2 + x1]);
    }
#pragma unroll
    for (int k = 0; k < NT; ++k) {
      const int t = lane + 32 * k;
      if (t < DD) win[p * STRIDE + t] = v[k];
    }
  }
  __syncthreads();
  const int p = threadIdx.x & (TP - 1), og = threadIdx.x >> 6;
  const int pix = pix0 + p;
  if (pix >= HW1) return;
  const float2 f = frac[p];
  const float* w = win + p * STRIDE;
  T* out = corr + (int64_t)n * NOUT * HW1 + pix;
#pragma unroll 3
  for (int o = og; o < NOUT; o += kCiThreads / TP) {
    const int a = o / RD, b = o - (o / RD) * RD;   // a along x, b along y
    const float v00 = w[b * D + a], v01 = w[(b + 1) * D + a];
    const float v10 = w[b * D + a + 1], v11 = w[(b + 1) * D + a + 1];
    const float val = (1.f - f.x) * (1.f - f.y) * v00 + (1.f - f.x) * f.y * v01 +
                      f.x * (1.f - f.y) * v10 + f.x * f.y * v11;
    out[(int64_t)o * HW1] = from_f<T>(val);
  }
}

template <typename T>
__global__ void __launch_bounds__(kCiThreads)
corr_index_bwd_kernel(const float* __restrict__ coords, const T* __restrict__ corr_grad,
                      T* __restrict__ volume_grad, int h1, int w1, int h2, int w2, int r, int tpix,
                      int stride) {
  extern __shared__ float4 smem4[];
  float4* geo = smem4;                                              // [tpix] dx, dy, x0, y0
  float* gwin = reinterpret_cast<float*>(smem4) + 4 * (size_t)tpix; // [tpix][stride] adjoint window

  const int n = blockIdx.y;
  const int HW1 = h1 * w1;
  const int64_t HW2 = (int64_t)h2 * w2;
  const int pix0 = blockIdx.x * tpix;
  const int npix = min(tpix, HW1 - pix0);
  const int D = 2 * r + 2;
  const int rd = 2 * r + 1;
  const int DD = D * D;

  for (int p = threadIdx.x; p < npix; p += kCiThreads) {
    const int pix = pix0 + p;
    const float cx = coords[((int64_t)n * 2 + 0) * HW1 + pix];
    const float cy = coords[((int64_t)n * 2 + 1) * HW1 + pix];
    const float fx = floorf(cx), fy = floorf(cy);
    geo[p] = make_float4(cx - fx, cy - fy, __int_as_float((int)fx - r), __int_as_float((int)fy - r));
  }
  __syncthreads();

  // window adjoint: G(i,j) gathers the <= 4 outputs that tapped (i,j)
  for (int idx = threadIdx.x; idx < npix * DD; idx += kCiThreads) {
    const int t = idx / npix;
    const int p = idx - t * npix;
    const float dx = geo[p].x, dy = geo[p].y;
    const int j = t / D;      // y index
    const int i = t - j * D;  // x index
    const T* g = corr_grad + (int64_t)n * rd * rd * HW1 + pix0 + p;
    float G = 0.f;
    if (i < rd && j < rd) G += (1.f - dx) * (1.f - dy) * to_f(g[(int64_t)(i * rd + j) * HW1]);
    if (i < rd && j > 0) G += (1.f - dx) * dy * to_f(g[(int64_t)(i * rd + j - 1) * HW1]);
    if (i > 0 && j < rd) G += dx * (1.f - dy) * to_f(g[(int64_t)((i - 1) * rd + j) * HW1]);
    if (i > 0 && j > 0) G += dx * dy * to_f(g[(int64_t)((i - 1) * rd + j - 1) * HW1]);
    gwin[p * stride + t] = G;
  }

  // zero the CTA's planes with 16-byte stores
  T* base = volume_grad + ((int64_t)n * HW1 + pix0) * HW2;
  const int64_t count = (int64_t)npix * HW2;
  {
    const uintptr_t addr = reinterpret_cast<uintptr_t>(base);
    int64_t head = (int64_t)(((16 - (addr & 15)) & 15) / sizeof(T));
    if (head > count) head = count;
    const int64_t nvec = (count - head) * (int64_t)sizeof(T) / 16;
    const int64_t tail0 = head + nvec * 16 / (int64_t)sizeof(T);
    for (int64_t k = threadIdx.x; k < head; k += kCiThreads) base[k] = from_f<T>(0.f);
    uint4* vb = reinterpret_cast<uint4*>(base + head);
    const uint4 z = make_uint4(0, 0, 0, 0);
    for (int64_t k = threadIdx.x; k < nvec; k += kCiThreads) vb[k] = z;
    for (int64_t k = tail0 + threadIdx.x; k < count; k += kCiThreads) base[k] = from_f<T>(0.f);
  }
  __syncthreads();

  // window values (distinct taps per pixel: no collisions)
  for (int idx = threadIdx.x; idx < npix * DD; idx += kCiThreads) {
    const int p = idx / DD;
    const int t = idx - p * DD;
    const float4 q = geo[p];
    const int j = t / D, i = t - (t / D) * D;
    const int x1 = __float_as_int(q.z) + i, y1 = __float_as_int(q.w) + j;
    if (x1 >= 0 && x1 < w2 && y1 >= 0 && y1 < h2)
      base[(int64_t)p * HW2 + (int64_t)y1 * w2 + x1] = from_f<T>(gwin[p * stride + t]);
  }
}

template <typename T>
static int launch_fwd(const void* volume, int64_t n, int h1, int w1, int h2, int w2, const float* coords,
                      int radius, void* corr, cudaStream_t stream) {
  const int HW1 = h1 * w1;
  if (radius == 3 || radius == 4) {
    dim3 grid((HW1 + 63) / 64, (unsigned)n);
    HS2_PROF("corr_index_fwd", stream);
    if (radius == 3)
      corr_index_fwd_r_kernel<T, 3><<<grid, kCiThreads, 0, stream>>>(static_cast<const T*>(volume), coords,
                                                                      static_cast<T*>(corr), h1, w1, h2, w2);
    else
      corr_index_fwd_r_kernel<T, 4><<<grid, kCiThreads, 0, stream>>>(static_cast<const T*>(volume), coords,
                                                                      static_cast<T*>(corr), h1, w1, h2, w2);
    HS2_LAUNCH_CHECK("corr_index_fwd_r_kernel");
    return HS2_OK;
  }
  const CiTile t = ci_tile(radius, 2 * radius + 1);
  dim3 grid((HW1 + t.tpix - 1) / t.tpix, (unsigned)n);
  if (t.smem > 48 * 1024)
    HS2_CUDA(cudaFuncSetAttribute(corr_index_fwd_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)t.smem));
  HS2_PROF("corr_index_fwd", stream);
  corr_index_fwd_kernel<T><<<grid, kCiThreads, t.smem, stream>>>(
      static_cast<const T*>(volume), coords, static_cast<T*>(corr), h1, w1, h2, w2, radius, t.tpix,
      t.stride);
  HS2_LAUNCH_CHECK("corr_index_fwd_kernel");
  return HS2_OK;
}

template <typename T>
static int launch_bwd(const float* coords, const void* corr_grad, int64_t n, int h1, int w1, int h2,
                      int w2, int radius, void* volume_grad, cudaStream_t stream) {
  const CiTile t = ci_tile(radius, 2 * radius + 1);
  const int HW1 = h1 * w1;
  dim3 grid((HW1 + t.tpix - 1) / t.tpix, (unsigned)n);
  if (t.smem > 48 * 1024)
    HS2_CUDA(cudaFuncSetAttribute(corr_index_bwd_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)t.smem));
  HS2_PROF("corr_index_bwd", stream);
  corr_index_bwd_kernel<T><<<grid, kCiThreads, t.smem, stream>>>(
      coords, static_cast<const T*>(corr_grad), static_cast<T*>(volume_grad), h1, w1, h2, w2, radius,
      t.tpix, t.stride);
  HS2_LAUNCH_CHECK("corr_index_bwd_kernel");
  return HS2_OK;
}

static int check_dims(const char* op, int64_t n, int h1, int w1, int h2, int w2, int radius) {
  if (n < 0 || h1 <= 0 || w1 <= 0 || h2 <= 0 || w2 <= 0 || radius < 0 || radius > 100 || n > 65535) {
    set_error("%s: bad sizes n=%lld h1=%d w1=%d h2=%d w2=%d r=%d", op, (long long)n, h1, w1, h2, w2,
              radius);
    return HS2_ERR_INVALID;
  }
  return HS2_OK;
}

}  // namespace hs2

extern "C" int hs2_corr_index_forward(const void* volume, int dtype, int64_t n, int h1, int w1, int h2,
                                      int w2, const float* coords, int radius, void* corr,
                                      hs2_stream_t stream) {
  using namespace hs2;
  int rc = check_dims("corr_index_forward", n, h1, w1, h2, w2, radius);
  if (rc) return rc;
  if (n == 0) return HS2_OK;
  if ((rc = bind_device(corr))) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  switch (dtype) {
    case HS2_F32: return launch_fwd<float>(volume, n, h1, w1, h2, w2, coords, radius, corr, s);
    case HS2_F16: return launch_fwd<__half>(volume, n, h1, w1, h2, w2, coords, radius, corr, s);
    case HS2_BF16: return launch_fwd<__nv_bfloat16>(volume, n, h1, w1, h2, w2, coords, radius, corr, s);
    case HS2_F64: return launch_fwd<double>(volume, n, h1, w1, h2, w2, coords, radius, corr, s);
  }
  set_error("corr_index_forward: unsupported dtype %d", dtype);
  return HS2_ERR_DTYPE;
}

extern "C" int hs2_corr_index_backward(const float* coords, const void* corr_grad, int dtype, int64_t n,
                                       int h1, int w1, int h2, int w2, int radius, void* volume_grad,
                                       hs2_stream_t stream) {
  using namespace hs2;
  int rc = check_dims("corr_index_backward", n, h1, w1, h2, w2, radius);
  if (rc) return rc;
  if (n == 0) return HS2_OK;
  if ((rc = bind_device(volume_grad))) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  switch (dtype) {
    case HS2_F32: return launch_bwd<float>(coords, corr_grad, n, h1, w1, h2, w2, radius, volume_grad, s);
    case HS2_F16: return launch_bwd<__half>(coords, corr_grad, n, h1, w1, h2, w2, radius, volume_grad, s);
    case HS2_BF16:
      return launch_bwd<__nv_bfloat16>(coords, corr_grad, n, h1, w1, h2, w2, radius, volume_grad, s);
    case HS2_F64: return launch_bwd<double>(coords, corr_grad, n, h1, w1, h2, w2, radius, volume_grad, s);
  }
  set_error("corr_index_backward: unsupported dtype %d", dtype);
  return HS2_ERR_DTYPE;
}
