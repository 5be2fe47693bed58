// altcorr_forward / altcorr_backward: correlation windows computed on the fly
// from feature maps, without materialising the all-pairs volume
// (reference: src/altcorr_kernel.cu:25-225).
//
// Forward: a CTA owns 32 consecutive pixels of one (batch, correlation m).
// Each work item (pixel, window row) forms the D = 2r+2 channel dot products of
// that row in registers (FP32 accumulation over the C channels), the D x D
// window lands in shared memory, and the bilinear blend writes the
// (2r+1)^2 outputs with consecutive threads on consecutive pixels.  The /4 /4
// feature scaling of the reference is applied once as 1/16 at the end.
//
// Backward: the adjoint of the bilinear blend is formed per window in shared
// memory, then fmap1/fmap2 gradients are accumulated with FP32 atomics (a
// frame may appear in several correlations).  `scale` multiplies every
// product; the reference operator corresponds to scale = 1.
#include "common.cuh"
#include "profile.cuh"

namespace hs2 {

constexpr int kAcThreads = 256;
constexpr int kAcPix = 32;    // pixels per CTA
constexpr int kAcTaps = 16;   // taps per register chunk

template <typename T>
__global__ void __launch_bounds__(kAcThreads)
altcorr_fwd_kernel(const T* __restrict__ fmap1, const T* __restrict__ fmap2, const float* __restrict__ coords,
                   const int64_t* __restrict__ ii, const int64_t* __restrict__ jj, T* __restrict__ corr,
                   int N1, int N2, int C, int H, int W, int H2, int W2, int M, int r, int stride,
                   int32_t* __restrict__ info) {
  extern __shared__ float4 smem4[];
  float4* geo = smem4;                                                   // [kAcPix]
  float* win = reinterpret_cast<float*>(smem4) + 4 * kAcPix;            // [kAcPix][stride]

  const int b = blockIdx.z;
  const int m = blockIdx.y;
  const int HW = H * W;
  const int64_t HW2 = (int64_t)H2 * W2;
  const int pix0 = blockIdx.x * kAcPix;
  const int D = 2 * r + 2;
  const int rd = 2 * r + 1;
  const int64_t ix = ii[m], jx = jj[m];
  const bool ok = ix >= 0 && ix < N1 && jx >= 0 && jx < N2;
  if (!ok && threadIdx.x == 0 && blockIdx.x == 0 && info) atomicOr(info, HS2_DEV_BAD_INDEX);

  const float* cx = coords + (((int64_t)b * M + m) * 2 + 0) * HW;
  const float* cy = coords + (((int64_t)b * M + m) * 2 + 1) * HW;
  for (int q = threadIdx.x; q < kAcPix; q += kAcThreads) {
    const int pix = min(pix0 + q, HW - 1);
    const float x = cx[pix], y = cy[pix];
    const float fx = floorf(x), fy = floorf(y);
    geo[q] = make_float4(x - fx, y - fy, __int_as_float((int)fx - r), __int_as_float((int)fy - r));
  }
  __syncthreads();

  const T* f1 = fmap1 + ((int64_t)b * N1 + (ok ? ix : 0)) * C * HW;
  const T* f2 = fmap2 + ((int64_t)b * N2 + (ok ? jx : 0)) * C * HW2;
  for (int item = threadIdx.x; item < kAcPix * D; item += kAcThreads) {
    const int py = item / kAcPix;
    const int q = item - py * kAcPix;
    const int pix = pix0 + q;
    float* wrow = win + q * stride + py * D;
    const float4 g = geo[q];
    const int y1 = __float_as_int(g.w) + py;
    const int xb = __float_as_int(g.z);
    const bool row_ok = ok && pix < HW && y1 >= 0 && y1 < H2;
    for (int c0 = 0; c0 < D; c0 += kAcTaps) {
      float acc[kAcTaps];
#pragma unroll
      for (int k = 0; k < kAcTaps; ++k) acc[k] = 0.f;
      if (row_ok) {
        const T* a = f1 + pix;
        const T* brow = f2 + (int64_t)y1 * W2;
        for (int c = 0; c < C; ++c) {
          const float av = to_f(a[(int64_t)c * HW]);
          const T* bc = brow + (int64_t)c * HW2;
#pragma unroll
          for (int k = 0; k < kAcTaps; ++k) {
            const int x1 = xb + c0 + k;
            if (c0 + k < D && x1 >= 0 && x1 < W2) acc[k] += av * to_f(bc[x1]);
          }
        }
      }
#pragma unroll
      for (int k = 0; k < kAcTaps; ++k)
        if (c0 + k < D) wrow[c0 + k] = acc[k] * 0.0625f;
    }
  }
  __syncthreads();

  const int nout = rd * rd;
  T* out = corr + ((int64_t)b * M + m) * nout * HW;
  for (int idx = threadIdx.x; idx < kAcPix * nout; idx += kAcThreads) {
    const int o = idx / kAcPix;
    const int q = idx - o * kAcPix;
    const int pix = pix0 + q;
    if (pix >= HW) continue;
    const int a = o / rd;      // x offset (dim 2 of the output)
    const int bb = o - a * rd; // y offset (dim 3 of the output)
    const float4 g = geo[q];
    const float* w = win + q * stride;
    const float v = (1.f - g.x) * (1.f - g.y) * w[bb * D + a] + g.x * (1.f - g.y) * w[bb * D + a + 1] +
                    (1.f - g.x) * g.y * w[(bb + 1) * D + a] + g.x * g.y * w[(bb + 1) * D + a + 1];
    out[(int64_t)o * HW + pix] = from_f<T>(v);
  }
}

template <typename T>
__global__ void __launch_bounds__(kAcThreads)
altcorr_bwd_kernel(const T* __restrict__ fmap1, const T* __restrict__ fmap2, const float* __restrict__ coords,
                   const int64_t* __restrict__ ii, const int64_t* __restrict__ jj, const float* __restrict__ grad,
                   float* __restrict__ g1, float* __restrict__ g2, int N1, int N2, int C, int H, int W,
                   int H2, int W2, int M, int r, int stride, float scale, int32_t* __restrict__ info) {
  extern __shared__ float4 smem4[];
  float4* geo = smem4;
  float* gw = reinterpret_cast<float*>(smem4) + 4 * kAcPix;

  const int b = blockIdx.z;
  const int m = blockIdx.y;
  const int HW = H * W;
  const int64_t HW2 = (int64_t)H2 * W2;
  const int pix0 = blockIdx.x * kAcPix;
  const int npix = min(kAcPix, HW - pix0);
  const int D = 2 * r + 2;
  const int DD = D * D;
  const int rd = 2 * r + 1;
  const int64_t ix = ii[m], jx = jj[m];
  if (!(ix >= 0 && ix < N1 && jx >= 0 && jx < N2)) {
    if (threadIdx.x == 0 && blockIdx.x == 0 && info) atomicOr(info, HS2_DEV_BAD_INDEX);
    return;
  }
  const float* cx = coords + (((int64_t)b * M + m) * 2 + 0) * HW;
  const float* cy = coords + (((int64_t)b * M + m) * 2 + 1) * HW;
  for (int q = threadIdx.x; q < npix; q += kAcThreads) {
    const float x = cx[pix0 + q], y = cy[pix0 + q];
    const float fx = floorf(x), fy = floorf(y);
    geo[q] = make_float4(x - fx, y - fy, __int_as_float((int)fx - r), __int_as_float((int)fy - r));
  }
  __syncthreads();
  // adjoint of the bilinear blend; grad layout [b, m, x-offset, y-offset, H, W]
  const float* gr = grad + ((int64_t)b * M + m) * rd * rd * HW + pix0;
  for (int idx = threadIdx.x; idx < npix * DD; idx += kAcThreads) {
    const int t = idx / npix;
    const int q = idx - t * npix;
    const int py = t / D, px = t - (t / D) * D;
    const float dx = geo[q].x, dy = geo[q].y;
    float G = 0.f;
    if (px < rd && py < rd) G += (1.f - dx) * (1.f - dy) * gr[(int64_t)(px * rd + py) * HW + q];
    if (px > 0 && py < rd) G += dx * (1.f - dy) * gr[(int64_t)((px - 1) * rd + py) * HW + q];
    if (px < rd && py > 0) G += (1.f - dx) * dy * gr[(int64_t)(px * rd + py - 1) * HW + q];
    if (px > 0 && py > 0) G += dx * dy * gr[(int64_t)((px - 1) * rd + py - 1) * HW + q];
    gw[q * stride + t] = G * scale;
  }
  __syncthreads();

  const T* f1 = fmap1 + ((int64_t)b * N1 + ix) * C * HW;
  const T* f2 = fmap2 + ((int64_t)b * N2 + jx) * C * HW2;
  float* o1 = g1 + ((int64_t)b * N1 + ix) * C * HW;
  float* o2 = g2 + ((int64_t)b * N2 + jx) * C * HW2;
  // fmap1 gradient: one (pixel, channel) per item, sum over the window
  for (int idx = threadIdx.x; idx < npix * C; idx += kAcThreads) {
    const int c = idx / npix;
    const int q = idx - c * npix;
    const float4 g = geo[q];
    const int xb = __float_as_int(g.z), yb = __float_as_int(g.w);
    const T* bc = f2 + (int64_t)c * HW2;
    float s = 0.f;
    for (int t = 0; t < DD; ++t) {
      const int py = t / D, px = t - (t / D) * D;
      const int x1 = xb + px, y1 = yb + py;
      if (x1 >= 0 && x1 < W2 && y1 >= 0 && y1 < H2) s += gw[q * stride + t] * to_f(bc[(int64_t)y1 * W2 + x1]);
    }
    atomicAdd(o1 + (int64_t)c * HW + pix0 + q, s);
  }
  // fmap2 gradient: one (pixel, tap) per item, loop over channels
  for (int idx = threadIdx.x; idx < npix * DD; idx += kAcThreads) {
    const int t = idx / npix;
    const int q = idx - t * npix;
    const float4 g = geo[q];
    const int py = t / D, px = t - (t / D) * D;
    const int x1 = __float_as_int(g.z) + px, y1 = __float_as_int(g.w) + py;
    if (x1 < 0 || x1 >= W2 || y1 < 0 || y1 >= H2) continue;
    const float G = gw[q * stride + t];
    if (G == 0.f) continue;
    const T* a = f1 + pix0 + q;
    float* dst = o2 + (int64_t)y1 * W2 + x1;
    for (int c = 0; c < C; ++c) atomicAdd(dst + (int64_t)c * HW2, G * to_f(a[(int64_t)c * HW]));
  }
}

// ---------------------------------------------------------------- packed forward ---
// Fast forward for 16-bit features.  Frames are first packed channel-last ([B, N, HW, C],
// one 2*C-byte row per pixel), so a window row of D positions is D contiguous rows: a
// warp computes one pixel's window row by row with lane (position q = lane % 8, channel
// group g = lane / 8) reading 16-byte chunks of its group's C/4 channels (the eight
// positions of a chunk step are 8 consecutive rows: coalesced), multiplying in FP32
// with f16/bf16 operands (fma.rn.f32.f16 / .bf16: exact products, FP32 sums) against
// the pixel's fmap1 row held in registers, and reducing the four groups by two
// shuffles.  The window lands in shared memory and the bilinear blend writes the
// outputs with consecutive threads on consecutive pixels, as in the direct kernel.

// channel-first [B, N, C, H, W] -> channel-last [B, N, HW, C] for the frames whose flag
// is set (every frame when flags is null); 32 pixels x C channels per CTA through
// shared memory
template <typename T>
__global__ void __launch_bounds__(kAcThreads)
altcorr_pack_kernel(const T* __restrict__ src, T* __restrict__ dst, const unsigned char* __restrict__ flags, int N,
                    int C, int HW) {
  __shared__ T tile[32][257];
  const int b = blockIdx.z, n = blockIdx.y;
  if (flags && !flags[n]) return;
  const int p0 = blockIdx.x * 32;
  const int np = min(32, HW - p0);
  const T* s = src + ((int64_t)b * N + n) * C * HW + p0;
  T* d = dst + (((int64_t)b * N + n) * HW + p0) * C;
  for (int idx = threadIdx.x; idx < C * 32; idx += kAcThreads) {
    const int c = idx >> 5, q = idx & 31;
    if (q < np) tile[q][c] = s[(int64_t)c * HW + q];
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < np * C; idx += kAcThreads) {
    const int q = idx / C, c = idx - q * C;
    d[(int64_t)q * C + c] = tile[q][c];
  }
}

__global__ void altcorr_flag_kernel(const int64_t* __restrict__ idx, int m, int n, unsigned char* __restrict__ flags) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < m; e += gridDim.x * blockDim.x) {
    const int64_t f = idx[e];
    if (f >= 0 && f < n) flags[f] = 1;
  }
}

template <typename T>
__device__ __forceinline__ void dot8(const uint4 a, const uint4 b, float& s0, float& s1);

template <>
__device__ __forceinline__ void dot8<__half>(const uint4 a, const uint4 b, float& s0, float& s1) {
  asm("{\n\t.reg .b16 al, ah, bl, bh;\n\t"
      "mov.b32 {al, ah}, %2;\n\tmov.b32 {bl, bh}, %6;\n\t"
      "fma.rn.f32.f16 %0, al, bl, %0;\n\tfma.rn.f32.f16 %1, ah, bh, %1;\n\t"
      "mov.b32 {al, ah}, %3;\n\tmov.b32 {bl, bh}, %7;\n\t"
      "fma.rn.f32.f16 %0, al, bl, %0;\n\tfma.rn.f32.f16 %1, ah, bh, %1;\n\t"
      "mov.b32 {al, ah}, %4;\n\tmov.b32 {bl, bh}, %8;\n\t"
      "fma.rn.f32.f16 %0, al, bl, %0;\n\tfma.rn.f32.f16 %1, ah, bh, %1;\n\t"
      "mov.b32 {al, ah}, %5;\n\tmov.b32 {bl, bh}, %9;\n\t"
      "fma.rn.f32.f16 %0, al, bl, %0;\n\tfma.rn.f32.f16 %1, ah, bh, %1;\n\t}"
      : "+f"(s0), "+f"(s1)
      : "r"(a.x), "r"(a.y), "r"(a.z), "r"(a.w), "r"(b.x), "r"(b.y), "r"(b.z), "r"(b.w));
}

template <>
__device__ __forceinline__ void dot8<__nv_bfloat16>(const uint4 a, const uint4 b, float& s0, float& s1) {
  asm("{\n\t.reg .b16 al, ah, bl, bh;\n\t"
      "mov.b32 {al, ah}, %2;\n\tmov.b32 {bl, bh}, %6;\n\t"
      "fma.rn.f32.bf16 %0, al, bl, %0;\n\tfma.rn.f32.bf16 %1, ah, bh, %1;\n\t"
      "mov.b32 {al, ah}, %3;\n\tmov.b32 {bl, bh}, %7;\n\t"
      "fma.rn.f32.bf16 %0, al, bl, %0;\n\tfma.rn.f32.bf16 %1, ah, bh, %1;\n\t"
      "mov.b32 {al, ah}, %4;\n\tmov.b32 {bl, bh}, %8;\n\t"
      "fma.rn.f32.bf16 %0, al, bl, %0;\n\tfma.rn.f32.bf16 %1, ah, bh, %1;\n\t"
      "mov.b32 {al, ah}, %5;\n\tmov.b32 {bl, bh}, %9;\n\t"
      "fma.rn.f32.bf16 %0, al, bl, %0;\n\tfma.rn.f32.bf16 %1, ah, bh, %1;\n\t}"
      : "+f"(s0), "+f"(s1)
      : "r"(a.x), "r"(a.y), "r"(a.z), "r"(a.w), "r"(b.x), "r"(b.y), "r"(b.z), "r"(b.w));
}

// NCH = C / 32: 16-byte chunks of a lane's channel group per position
template <typename T, int NCH>
__global__ void __launch_bounds__(kAcThreads)
altcorr_fwd_packed_kernel(const T* __restrict__ p1, const T* __restrict__ p2, const float* __restrict__ coords,
                          const int64_t* __restrict__ ii, const int64_t* __restrict__ jj, T* __restrict__ corr,
                          int N1, int N2, int H, int W, int H2, int W2, int M, int r, int stride,
                          int32_t* __restrict__ info) {
  constexpr int C = 32 * NCH;
  extern __shared__ float4 smem4[];
  float4* geo = smem4;                                                   // [kAcPix]
  float* win = reinterpret_cast<float*>(smem4) + 4 * kAcPix;            // [kAcPix][stride]
  const int b = blockIdx.z, m = blockIdx.y;
  const int HW = H * W;
  const int pix0 = blockIdx.x * kAcPix;
  const int npix = min(kAcPix, HW - pix0);
  const int D = 2 * r + 2, rd = 2 * r + 1;
  const int64_t ix = ii[m], jx = jj[m];
  const bool ok = ix >= 0 && ix < N1 && jx >= 0 && jx < N2;
  if (!ok && threadIdx.x == 0 && blockIdx.x == 0 && info) atomicOr(info, HS2_DEV_BAD_INDEX);
  const float* cx = coords + (((int64_t)b * M + m) * 2 + 0) * HW;
  const float* cy = coords + (((int64_t)b * M + m) * 2 + 1) * HW;
  for (int q = threadIdx.x; q < npix; q += kAcThreads) {
    const float x = cx[pix0 + q], y = cy[pix0 + q];
    const float fx = floorf(x), fy = floorf(y);
    geo[q] = make_float4(x - fx, y - fy, __int_as_float((int)fx - r), __int_as_float((int)fy - r));
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int pq = lane & 7, g = lane >> 3;
  const T* f1 = p1 + ((int64_t)b * N1 + (ok ? ix : 0)) * HW * C;
  const T* f2 = p2 + ((int64_t)b * N2 + (ok ? jx : 0)) * (int64_t)H2 * W2 * C;
  for (int q = warp; q < npix; q += kAcThreads / 32) {
    const float4 gq = geo[q];
    const int xb = __float_as_int(gq.z), yb = __float_as_int(gq.w);
    const uint4* a = reinterpret_cast<const uint4*>(f1 + (int64_t)(pix0 + q) * C) + g * NCH;
    uint4 av[NCH];
#pragma unroll
    for (int k = 0; k < NCH; ++k) av[k] = __ldg(a + k);
    float* wq = win + q * stride;
    for (int py = 0; py < D; ++py) {
      const int y1 = yb + py;
      for (int pc = 0; pc < D; pc += 8) {
        const int px = pc + pq, x1 = xb + px;
        float s0 = 0.f, s1 = 0.f;
        if (ok && px < D && y1 >= 0 && y1 < H2 && x1 >= 0 && x1 < W2) {
          const uint4* bp = reinterpret_cast<const uint4*>(f2 + ((int64_t)y1 * W2 + x1) * C) + g * NCH;
#pragma unroll
          for (int k = 0; k < NCH; ++k) dot8<T>(av[k], __ldg(bp + k), s0, s1);
        }
        float sv = s0 + s1;
        sv += __shfl_xor_sync(0xffffffffu, sv, 8);
        sv += __shfl_xor_sync(0xffffffffu, sv, 16);
        if (g == 0 && px < D) wq[py * D + px] = sv * 0.0625f;
      }
    }
  }
  __syncthreads();
  const int nout = rd * rd;
  T* out = corr + ((int64_t)b * M + m) * nout * HW;
  for (int idx = threadIdx.x; idx < npix * nout; idx += kAcThreads) {
    const int o = idx / npix;
    const int q = idx - o * npix;
    const int a = o / rd;      // x offset (dim 2 of the output)
    const int bb = o - a * rd; // y offset (dim 3 of the output)
    const float4 gq = geo[q];
    const float* w = win + q * stride;
    const float v = (1.f - gq.x) * (1.f - gq.y) * w[bb * D + a] + gq.x * (1.f - gq.y) * w[bb * D + a + 1] +
                    (1.f - gq.x) * gq.y * w[(bb + 1) * D + a] + gq.x * gq.y * w[(bb + 1) * D + a + 1];
    out[(int64_t)o * HW + pix0 + q] = from_f<T>(v);
  }
}

// ------------------------------------------------------------ tile forward ---
// Dense local correlation on the tensor cores for C = 128 channels.  A CTA owns an 8x8
// block of pixels of one edge.  The union of the block's D x D windows is a box of
// bw x bh target positions (about 19 x 19 at 43x77 for reprojected coordinates); when it
// holds at most kAtMaxPos positions the CTA stages the 64 source rows and the box's
// rows (channel-last, 16-byte cp.async) in shared memory and computes the full
// 64 x (bw bh) product with mma.sync m16n8k16 (16-bit operands, FP32 accumulation:
// exact products, FP32 sums), then every output tap reads its four window values from
// that product.  The product is 5-6x the taps actually needed, but it runs on the
// tensor pipe and every target row is read once per block instead of once per pixel
// and window row.  Blocks whose box is larger (coordinates scattered across the image)
// fall back to the warp-per-pixel channel-last computation, so any input is correct.
// mma.sync rather than tcgen05: the B operand is a data-dependent gathered box of
// up to 384 rows and M is 64 (tcgen05 wants M = 128, i.e. a 16x8 block whose box no
// longer fits next to its accumulator staging), and the kernel is bounded by the
// staging and the gather epilogue, not by the tensor pipe.
constexpr int kAtSide = 8;
constexpr int kAtPix = kAtSide * kAtSide;
constexpr int kAtThreads = 512;        // 16 warps: 4 m-tiles x 4 n-tile phases
constexpr int kAtMaxPos = 384;
constexpr int kAtLd = 136;             // halves per staged row: 128 channels + 16 bytes of padding
constexpr int kAtDLd = kAtMaxPos + 4;  // floats per row of the staged product
constexpr size_t kAtSmem = (size_t)kAtPix * kAtLd * 2 + (size_t)kAtMaxPos * kAtLd * 2 +
                           (size_t)kAtPix * kAtDLd * 4 + kAtPix * 16 + 128;

template <typename T>
__device__ __forceinline__ void mma16816(float* d, const uint32_t* a, uint32_t b0, uint32_t b1);

template <>
__device__ __forceinline__ void mma16816<__half>(float* d, const uint32_t* a, uint32_t b0, uint32_t b1) {
  asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
               "{%0,%1,%2,%3};"
               : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
               : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

template <>
__device__ __forceinline__ void mma16816<__nv_bfloat16>(float* d, const uint32_t* a, uint32_t b0, uint32_t b1) {
  asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
               "{%0,%1,%2,%3};"
               : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
               : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ void ldsm_x4(uint32_t* r, uint32_t addr) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]) : "r"(addr));
}
__device__ __forceinline__ void ldsm_x2(uint32_t& r0, uint32_t& r1, uint32_t addr) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x2.shared.b16 {%0,%1}, [%2];" : "=r"(r0), "=r"(r1) : "r"(addr));
}
__device__ __forceinline__ uint32_t at_smem(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void at_cp16(uint32_t dst, const void* src, uint32_t bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}

// Arguments of the tile kernel.  altcorr: window coordinates read from `coords`
// [B][M][2][H][W], target features p2[0], output [B][M][2r+1][2r+1][H][W].  Fused
// reprojection + lookup (kFused): blockIdx.z is the level, coordinates are the
// reprojection of frame ii's pixels into frame jj (poses, disps, intrinsics; the float
// formula of corr_fused.cu) scaled by 2^-level, target features p2[level], output
// [M][levels * (2r+1)^2][H][W], and the level-0 coordinates optionally to coords_out.
struct AtArgs {
  const void* p1;
  const void* p2[4];
  const float* coords;
  const int64_t* ii;
  const int64_t* jj;
  void* corr;
  int N1, N2, H, W, H2, W2, M, r, levels;
  int32_t* info;
  const float* poses;
  const float* disps;
  const float* intr;
  int64_t num_poses, num_disps;
  float* coords_out;
};

template <typename T, bool kFused>
__global__ void __launch_bounds__(kAtThreads, 1)
altcorr_fwd_tile_kernel(const __grid_constant__ AtArgs A) {
  constexpr int C = 128;
  const int H = A.H, W = A.W, r = A.r, M = A.M, N1 = A.N1, N2 = A.N2;
  const int lvl = kFused ? (int)blockIdx.z : 0;
  const int H2 = kFused ? H >> lvl : A.H2, W2 = kFused ? W >> lvl : A.W2;
  const int64_t* __restrict__ ii = A.ii;
  const int64_t* __restrict__ jj = A.jj;
  const T* __restrict__ p1 = static_cast<const T*>(A.p1);
  const T* __restrict__ p2 = static_cast<const T*>(A.p2[kFused ? lvl : 0]);
  __shared__ float G[12];   // fused: R (row-major) then t of Gij
  extern __shared__ __align__(16) uint8_t at_raw[];
  T* As = reinterpret_cast<T*>(at_raw);                                         // [64][kAtLd]
  T* Bs = As + kAtPix * kAtLd;                                                  // [kAtMaxPos][kAtLd]
  float* Ds = reinterpret_cast<float*>(Bs + kAtMaxPos * kAtLd);                 // [64][kAtDLd]
  float4* geo = reinterpret_cast<float4*>(Ds + kAtPix * kAtDLd);               // [64]
  // box[12]: x0 min, y0 min, x0 max, y0 max of the whole block, then of its top and bottom
  // halves (rows 0-3, 4-7); reg[8]: per region bx0, by0, bw, mode (0 empty, 1 box, 2 window)
  int* box = reinterpret_cast<int*>(geo + kAtPix);
  int* reg = box + 12;
  const int b = kFused ? 0 : (int)blockIdx.z, m = blockIdx.y;
  const int HW = H * W;
  const int ntx = (W + kAtSide - 1) / kAtSide;
  const int tx0 = (blockIdx.x % ntx) * kAtSide, ty0 = (blockIdx.x / ntx) * kAtSide;
  const int D = 2 * r + 2, rd = 2 * r + 1;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t ix = ii[m], jx = jj[m];
  const bool ok = kFused ? (ix >= 0 && jx >= 0 && ix < N1 && jx < N1 && ix < A.num_poses && jx < A.num_poses &&
                            ix < A.num_disps)
                         : (ix >= 0 && ix < N1 && jx >= 0 && jx < N2);
  if (!ok && tid == 0 && blockIdx.x == 0 && lvl == 0 && A.info) atomicOr(A.info, HS2_DEV_BAD_INDEX);
  if (tid < 12) box[tid] = (tid & 3) < 2 ? 0x7fffffff : -0x7fffffff;
  if (kFused && tid == 0) {
    float t[3], q[4];
    if (ok) {
      relative_pose(A.poses + 7 * ix, A.poses + 7 * ix + 3, A.poses + 7 * jx, A.poses + 7 * jx + 3, t, q);
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
  if (tid < kAtPix) {
    const int px = tx0 + (tid & 7), py = ty0 + (tid >> 3);
    if (px < W && py < H) {
      float x, y;
      if (kFused) {
        const float fx = A.intr[0], fy = A.intr[1], cx = A.intr[2], cy = A.intr[3];
        const int pix = py * W + px;
        const float d = ok ? A.disps[ix * HW + pix] : 0.f;
        const float X = (px - cx) / fx, Y = (py - cy) / fy;
        const float P0 = G[0] * X + G[1] * Y + G[2] + G[9] * d;
        const float P1 = G[3] * X + G[4] * Y + G[5] + G[10] * d;
        const float P2 = G[6] * X + G[7] * Y + G[8] + G[11] * d;
        const float xc = fx * (P0 / P2) + cx, yc = fy * (P1 / P2) + cy;
        if (lvl == 0 && A.coords_out) {
          A.coords_out[((int64_t)m * HW + pix) * 2 + 0] = xc;
          A.coords_out[((int64_t)m * HW + pix) * 2 + 1] = yc;
        }
        const float scale = 1.0f / (float)(1 << lvl);
        x = xc * scale;
        y = yc * scale;
      } else {
        x = A.coords[(((int64_t)b * M + m) * 2 + 0) * HW + py * W + px];
        y = A.coords[(((int64_t)b * M + m) * 2 + 1) * HW + py * W + px];
      }
      const float fx = floorf(x), fy = floorf(y);
      const int x0 = (int)fx - r, y0 = (int)fy - r;
      geo[tid] = make_float4(x - fx, y - fy, __int_as_float(x0), __int_as_float(y0));
      int* bh = box + 4 * (1 + (tid >> 5));
      atomicMin(&box[0], x0);
      atomicMin(&box[1], y0);
      atomicMax(&box[2], x0);
      atomicMax(&box[3], y0);
      atomicMin(&bh[0], x0);
      atomicMin(&bh[1], y0);
      atomicMax(&bh[2], x0);
      atomicMax(&bh[3], y0);
    }
  }
  __syncthreads();
  // regions: the whole block when its box (window positions inside the target only) fits
  // the staging area, else its two halves, each staged if it fits and computed per pixel
  // otherwise; an empty box means all of the region's taps are 0
  auto box_of = [&](const int* bb, int& x0, int& y0, int& w, int& h) {
    if (bb[0] > bb[2]) {   // no pixel in the region
      x0 = y0 = w = h = 0;
      return;
    }
    x0 = max(bb[0], 0);
    y0 = max(bb[1], 0);
    w = min(min(bb[2], W2) + D, W2) - x0;
    h = min(min(bb[3], H2) + D, H2) - y0;
    if (w <= 0 || h <= 0) w = h = 0;
  };
  int fx0, fy0, fw, fh;
  box_of(box, fx0, fy0, fw, fh);
  const int nreg = (ok && fw * fh > kAtMaxPos) ? 2 : 1;
  const T* f1 = p1 + ((int64_t)b * N1 + (ok ? ix : 0)) * HW * C;
  const T* f2 = p2 + ((int64_t)b * N2 + (ok ? jx : 0)) * (int64_t)H2 * W2 * C;
  const uint32_t sA = at_smem(As), sB = at_smem(Bs);
  bool a_staged = false;
  for (int rg = 0; rg < nreg; ++rg) {
    int bx0, by0, bw, bh;
    if (nreg == 1) {
      bx0 = fx0, by0 = fy0, bw = fw, bh = fh;
    } else {
      box_of(box + 4 * (1 + rg), bx0, by0, bw, bh);
    }
    const int npos = ok ? bw * bh : 0;
    const int mode = npos == 0 ? 0 : (npos <= kAtMaxPos ? 1 : 2);
    const int r0 = nreg == 1 ? 0 : 32 * rg, nrows = nreg == 1 ? kAtPix : 32;
    if (tid == 0) {
      reg[4 * rg + 0] = bx0;
      reg[4 * rg + 1] = by0;
      reg[4 * rg + 2] = bw;
      reg[4 * rg + 3] = mode;
    }
    if (mode == 1) {
      const int npad = (npos + 7) & ~7;
      const int arows = a_staged ? 0 : kAtPix;
      // n / bw without an integer division: for the staged box (n, bw <= 384) (n + 0.5) / bw
      // stays at least 0.5 / bw from an integer, far beyond the float rounding
      const float inv_bw = 1.f / (float)bw;
      // one item = a quarter row (four 16-byte copies): the row's address is formed once
      for (int idx = tid; idx < (arows + npad) * 4; idx += kAtThreads) {
        const int row = idx >> 2, ch0 = (idx & 3) * 32;
        const T* src;
        uint32_t dst, bytes;
        if (row < arows) {
          const int px = tx0 + (row & 7), py = ty0 + (row >> 3);
          const bool live = px < W && py < H;
          src = live ? f1 + (int64_t)(py * W + px) * C + ch0 : f1;
          bytes = live ? 16u : 0u;
          dst = sA + (uint32_t)(row * kAtLd + ch0) * 2u;
        } else {
          const int n = row - arows;
          const bool live = n < npos;
          const int qy = __float2int_rz(((float)n + 0.5f) * inv_bw);
          src = live ? f2 + ((int64_t)(by0 + qy) * W2 + bx0 + n - qy * bw) * C + ch0 : f2;
          bytes = live ? 16u : 0u;
          dst = sB + (uint32_t)(n * kAtLd + ch0) * 2u;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) at_cp16(dst + 16u * u, bytes ? (const void*)(src + 8 * u) : (const void*)src, bytes);
      }
      a_staged = true;
      asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
      __syncthreads();
      // warp: one of the region's m-tiles (16 pixels), n-tiles strided over the other warps
      const int nmt = nrows >> 4;
      const int mt = (r0 >> 4) + warp % nmt;
      const int nstep = (kAtThreads / 32) / nmt;   // 4 (whole block) or 8 (half) n-tile phases
      uint32_t af[8][4];
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const int rr = (lane & 7) + 8 * ((lane >> 3) & 1), kc = 16 * k + 8 * (lane >> 4);
        ldsm_x4(af[k], sA + (uint32_t)((16 * mt + rr) * kAtLd + kc) * 2u);
      }
      const int ntile = npad >> 3;
      for (int nt = warp / nmt; nt < ntile; nt += nstep) {
        float d[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          uint32_t b0, b1;
          const int nr = 8 * nt + (lane & 7), kc = 16 * k + 8 * ((lane >> 3) & 1);
          ldsm_x2(b0, b1, sB + (uint32_t)(nr * kAtLd + kc) * 2u);
          mma16816<T>(d, af[k], b0, b1);
        }
        const int row = 16 * mt + (lane >> 2), col = 8 * nt + 2 * (lane & 3);
        *reinterpret_cast<float2*>(&Ds[row * kAtDLd + col]) = make_float2(d[0], d[1]);
        *reinterpret_cast<float2*>(&Ds[(row + 8) * kAtDLd + col]) = make_float2(d[2], d[3]);
      }
      __syncthreads();   // the staging area is reused by the next region
    } else if (mode == 2) {
      // scattered coordinates: per pixel, one warp computes the D x D window (lanes: 8
      // positions x 4 channel groups of 32), stored window-major in the pixel's row of Ds
      const int pq = lane & 7, g = lane >> 3;
      for (int q = r0 + warp; q < r0 + nrows; q += kAtThreads / 32) {
        const int px = tx0 + (q & 7), py = ty0 + (q >> 3);
        if (px >= W || py >= H) continue;
        const float4 gq = geo[q];
        const int xb = __float_as_int(gq.z), yb = __float_as_int(gq.w);
        const uint4* a = reinterpret_cast<const uint4*>(f1 + (int64_t)(py * W + px) * C) + g * 4;
        uint4 av[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) av[k] = __ldg(a + k);
        for (int wy = 0; wy < D; ++wy) {
          const int y1 = yb + wy;
          for (int pc = 0; pc < D; pc += 8) {
            const int wx = pc + pq, x1 = xb + wx;
            float s0 = 0.f, s1 = 0.f;
            if (wx < D && y1 >= 0 && y1 < H2 && x1 >= 0 && x1 < W2) {
              const uint4* bp = reinterpret_cast<const uint4*>(f2 + ((int64_t)y1 * W2 + x1) * C) + g * 4;
#pragma unroll
              for (int k = 0; k < 4; ++k) dot8<T>(av[k], __ldg(bp + k), s0, s1);
            }
            float sv = s0 + s1;
            sv += __shfl_xor_sync(0xffffffffu, sv, 8);
            sv += __shfl_xor_sync(0xffffffffu, sv, 16);
            if (g == 0 && wx < D) Ds[q * kAtDLd + wy * D + wx] = sv;
          }
        }
      }
    }
  }
  __syncthreads();
  // bilinear blend: thread (pixel q, x offset a) walks the window rows, keeping the two
  // values of the previous row, so each output reads two new window values; taps outside
  // the target are 0
  const int nout = rd * rd;
  T* out = static_cast<T*>(A.corr) + (kFused ? ((int64_t)m * A.levels + lvl) : ((int64_t)b * M + m)) * nout * HW;
  for (int idx = tid; idx < kAtPix * rd; idx += kAtThreads) {
    const int q = idx & 63, a = idx >> 6;
    const int px = tx0 + (q & 7), py = ty0 + (q >> 3);
    if (px >= W || py >= H) continue;
    const int* rq = reg + 4 * (nreg == 1 ? 0 : q >> 5);
    const int mode = rq[3];
    T* oq = out + (int64_t)(a * rd) * HW + py * W + px;
    if (mode == 0) {
      for (int bb = 0; bb < rd; ++bb) oq[(int64_t)bb * HW] = from_f<T>(0.f);
      continue;
    }
    const float4 gq = geo[q];
    const int xb = __float_as_int(gq.z), yb = __float_as_int(gq.w);
    const int x1 = xb + a;
    const bool va = x1 >= 0 && x1 < W2, vb = x1 + 1 >= 0 && x1 + 1 < W2;
    // row-major addressing of the window values: the staged box (mode 1) or the pixel's own
    // D x D window (mode 2)
    const int rs = mode == 1 ? rq[2] : D;
    const float* dq = Ds + q * kAtDLd + (mode == 1 ? (yb - rq[1]) * rs + (x1 - rq[0]) : a);
    const float w00 = (1.f - gq.x) * (1.f - gq.y), w01 = gq.x * (1.f - gq.y);
    const float w10 = (1.f - gq.x) * gq.y, w11 = gq.x * gq.y;
    float t0 = 0.f, t1 = 0.f;
    for (int wy = 0; wy <= rd; ++wy) {
      const int y1 = yb + wy;
      const bool vy = y1 >= 0 && y1 < H2;
      const float* row = dq + wy * rs;
      const float u0 = (vy && va) ? row[0] : 0.f, u1 = (vy && vb) ? row[1] : 0.f;
      if (wy > 0)
        oq[(int64_t)(wy - 1) * HW] = from_f<T>((w00 * t0 + w01 * t1 + w10 * u0 + w11 * u1) * 0.0625f);
      t0 = u0;
      t1 = u1;
    }
  }
}

template <typename T>
__global__ void cast_from_f32_kernel(const float* __restrict__ src, T* __restrict__ dst, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = from_f<T>(src[i]);
}

static int ac_stride(int radius) {
  const int D = 2 * radius + 2;
  int s = D * D;
  if ((s & 1) == 0) s += 1;
  return s;
}

static int ac_check(const char* op, int b, int n1, int n2, int c, int h, int w, int h2, int w2, int m,
                    int radius) {
  if (b < 0 || n1 < 0 || n2 < 0 || c <= 0 || h <= 0 || w <= 0 || h2 <= 0 || w2 <= 0 || m < 0 ||
      radius < 0 || radius > 30 || m > 65535 || b > 65535) {
    set_error("%s: bad sizes b=%d n1=%d n2=%d c=%d h=%d w=%d h2=%d w2=%d m=%d r=%d", op, b, n1, n2, c, h, w,
              h2, w2, m, radius);
    return HS2_ERR_INVALID;
  }
  return HS2_OK;
}

template <typename T>
static int ac_fwd(const void* fmap1, const void* fmap2, int b, int n1, int n2, int c, int h, int w, int h2,
                  int w2, const float* coords, const int64_t* ii, const int64_t* jj, int m, int radius,
                  void* corr, int32_t* info, cudaStream_t s) {
  const int stride = ac_stride(radius);
  const size_t smem = (size_t)kAcPix * (stride * 4 + 16);
  if (smem > 48 * 1024)
    HS2_CUDA(cudaFuncSetAttribute(altcorr_fwd_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  dim3 grid((h * w + kAcPix - 1) / kAcPix, m, b);
  HS2_PROF("altcorr_fwd", s);
  altcorr_fwd_kernel<T><<<grid, kAcThreads, smem, s>>>(
      static_cast<const T*>(fmap1), static_cast<const T*>(fmap2), coords, ii, jj, static_cast<T*>(corr), n1,
      n2, c, h, w, h2, w2, m, radius, stride, info);
  HS2_LAUNCH_CHECK("altcorr_fwd_kernel");
  return HS2_OK;
}

template <typename T>
static int ac_bwd(const void* fmap1, const void* fmap2, int b, int n1, int n2, int c, int h, int w, int h2,
                  int w2, const float* coords, const int64_t* ii, const int64_t* jj, int m, const float* grad,
                  int radius, float scale, void* g1, void* g2, int32_t* info, void* ws, cudaStream_t s) {
  const int64_t n1el = (int64_t)b * n1 * c * h * w;
  const int64_t n2el = (int64_t)b * n2 * c * h2 * w2;
  float* a1 = std::is_same<T, float>::value ? static_cast<float*>(g1) : static_cast<float*>(ws);
  float* a2 = std::is_same<T, float>::value ? static_cast<float*>(g2) : static_cast<float*>(ws) + n1el;
  HS2_CUDA(cudaMemsetAsync(a1, 0, n1el * sizeof(float), s));
  HS2_CUDA(cudaMemsetAsync(a2, 0, n2el * sizeof(float), s));
  const int stride = ac_stride(radius);
  const size_t smem = (size_t)kAcPix * (stride * 4 + 16);
  if (smem > 48 * 1024)
    HS2_CUDA(cudaFuncSetAttribute(altcorr_bwd_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  if (m > 0 && b > 0) {
    dim3 grid((h * w + kAcPix - 1) / kAcPix, m, b);
    HS2_PROF("altcorr_bwd", s);
    altcorr_bwd_kernel<T><<<grid, kAcThreads, smem, s>>>(
        static_cast<const T*>(fmap1), static_cast<const T*>(fmap2), coords, ii, jj, grad, a1, a2, n1, n2, c, h,
        w, h2, w2, m, radius, stride, scale, info);
    HS2_LAUNCH_CHECK("altcorr_bwd_kernel");
  }
  if (!std::is_same<T, float>::value) {
    if (n1el) {
      cast_from_f32_kernel<T><<<1184, 256, 0, s>>>(a1, static_cast<T*>(g1), n1el);
      HS2_LAUNCH_CHECK("cast_from_f32_kernel");
    }
    if (n2el) {
      cast_from_f32_kernel<T><<<1184, 256, 0, s>>>(a2, static_cast<T*>(g2), n2el);
      HS2_LAUNCH_CHECK("cast_from_f32_kernel");
    }
  }
  return HS2_OK;
}

template <typename T>
static int ac_pack(const void* fmap, int b, int n, int c, int h, int w, const int64_t* frames, int num_frames,
                   void* packed, unsigned char* flags, cudaStream_t s) {
  if (frames) {
    HS2_CUDA(cudaMemsetAsync(flags, 0, (size_t)n, s));
    if (num_frames > 0) {
      altcorr_flag_kernel<<<(num_frames + 255) / 256, 256, 0, s>>>(frames, num_frames, n, flags);
      HS2_LAUNCH_CHECK("altcorr_flag_kernel");
    }
  }
  dim3 grid((h * w + 31) / 32, n, b);
  HS2_PROF("altcorr_pack", s);
  altcorr_pack_kernel<T><<<grid, kAcThreads, 0, s>>>(static_cast<const T*>(fmap), static_cast<T*>(packed),
                                                     frames ? flags : nullptr, n, c, h * w);
  HS2_LAUNCH_CHECK("altcorr_pack_kernel");
  return HS2_OK;
}

template <typename T, int NCH>
static int ac_fwd_packed_n(const void* p1, const void* p2, int b, int n1, int n2, int h, int w, int h2, int w2,
                           const float* coords, const int64_t* ii, const int64_t* jj, int m, int radius, void* corr,
                           int32_t* info, cudaStream_t s) {
  const int stride = ac_stride(radius);
  const size_t smem = (size_t)kAcPix * (stride * 4 + 16);
  if (smem > 48 * 1024)
    HS2_CUDA(cudaFuncSetAttribute(altcorr_fwd_packed_kernel<T, NCH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem));
  dim3 grid((h * w + kAcPix - 1) / kAcPix, m, b);
  HS2_PROF("altcorr_fwd_packed", s);
  altcorr_fwd_packed_kernel<T, NCH><<<grid, kAcThreads, smem, s>>>(
      static_cast<const T*>(p1), static_cast<const T*>(p2), coords, ii, jj, static_cast<T*>(corr), n1, n2, h, w, h2,
      w2, m, radius, stride, info);
  HS2_LAUNCH_CHECK("altcorr_fwd_packed_kernel");
  return HS2_OK;
}

template <typename T, bool kFused>
static int at_prepare() {
  static DeviceOnce once;
  int dev = 0;
  HS2_CUDA(cudaGetDevice(&dev));
  return once.run(dev, [&]() -> int {
    HS2_CUDA(cudaFuncSetAttribute(altcorr_fwd_tile_kernel<T, kFused>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)kAtSmem));
    return HS2_OK;
  });
}

template <typename T>
static int ac_fwd_packed(const void* p1, const void* p2, int b, int n1, int n2, int c, int h, int w, int h2, int w2,
                         const float* coords, const int64_t* ii, const int64_t* jj, int m, int radius, void* corr,
                         int32_t* info, cudaStream_t s) {
  switch (c) {
    case 32: return ac_fwd_packed_n<T, 1>(p1, p2, b, n1, n2, h, w, h2, w2, coords, ii, jj, m, radius, corr, info, s);
    case 64: return ac_fwd_packed_n<T, 2>(p1, p2, b, n1, n2, h, w, h2, w2, coords, ii, jj, m, radius, corr, info, s);
    case 128: {
      if (radius <= 8) {   // windows up to 18 x 18 taps
        int rc = at_prepare<T, false>();
        if (rc) return rc;
        AtArgs a{};
        a.p1 = p1;
        a.p2[0] = p2;
        a.coords = coords;
        a.ii = ii;
        a.jj = jj;
        a.corr = corr;
        a.N1 = n1, a.N2 = n2, a.H = h, a.W = w, a.H2 = h2, a.W2 = w2, a.M = m, a.r = radius, a.levels = 1;
        a.info = info;
        const int ntiles = ((w + kAtSide - 1) / kAtSide) * ((h + kAtSide - 1) / kAtSide);
        dim3 grid(ntiles, m, b);
        HS2_PROF("altcorr_fwd_tile", s);
        altcorr_fwd_tile_kernel<T, false><<<grid, kAtThreads, kAtSmem, s>>>(a);
        HS2_LAUNCH_CHECK("altcorr_fwd_tile_kernel");
        return HS2_OK;
      }
      return ac_fwd_packed_n<T, 4>(p1, p2, b, n1, n2, h, w, h2, w2, coords, ii, jj, m, radius, corr, info, s);
    }
    case 256: return ac_fwd_packed_n<T, 8>(p1, p2, b, n1, n2, h, w, h2, w2, coords, ii, jj, m, radius, corr, info, s);
  }
  set_error("altcorr_forward_packed: channels must be 32, 64, 128 or 256 (got %d)", c);
  return HS2_ERR_INVALID;
}

static size_t ac_packed_bytes(int dtype, int b, int n, int c, int h, int w) {
  return (size_t)b * n * h * w * c * (dtype == HS2_F16 || dtype == HS2_BF16 ? 2 : 0);
}

}  // namespace hs2

extern "C" int hs2_altcorr_pack_workspace_size(int dtype, int b, int n, int c, int h, int w, size_t* bytes) {
  using namespace hs2;
  if (!bytes) {
    set_error("altcorr_pack_workspace_size: null output");
    return HS2_ERR_INVALID;
  }
  if (dtype != HS2_F16 && dtype != HS2_BF16) {
    set_error("altcorr_pack: float16 or bfloat16 features only (dtype %d)", dtype);
    return HS2_ERR_DTYPE;
  }
  if (b < 0 || n < 0 || c <= 0 || c > 256 || h <= 0 || w <= 0 || b > 65535 || n > 65535) {
    set_error("altcorr_pack: bad sizes b=%d n=%d c=%d h=%d w=%d", b, n, c, h, w);
    return HS2_ERR_INVALID;
  }
  *bytes = ((ac_packed_bytes(dtype, b, n, c, h, w) + 255) & ~(size_t)255) + (size_t)n + 256;
  return HS2_OK;
}

extern "C" int hs2_altcorr_pack(const void* fmap, int dtype, int b, int n, int c, int h, int w,
                                const int64_t* frames, int num_frames, void* workspace, size_t workspace_bytes,
                                hs2_stream_t stream) {
  using namespace hs2;
  size_t need = 0;
  int rc = hs2_altcorr_pack_workspace_size(dtype, b, n, c, h, w, &need);
  if (rc) return rc;
  if (!workspace || workspace_bytes < need) {
    set_error("altcorr_pack: workspace of %zu bytes required", need);
    return HS2_ERR_WORKSPACE;
  }
  if (num_frames < 0 || (num_frames > 0 && !frames)) {
    set_error("altcorr_pack: bad frame list (%d)", num_frames);
    return HS2_ERR_INVALID;
  }
  if (b == 0 || n == 0) return HS2_OK;
  if ((rc = bind_device(workspace))) return rc;
  unsigned char* flags = static_cast<unsigned char*>(workspace) +
                         ((ac_packed_bytes(dtype, b, n, c, h, w) + 255) & ~(size_t)255);
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == HS2_F16) return ac_pack<__half>(fmap, b, n, c, h, w, frames, num_frames, workspace, flags, s);
  return ac_pack<__nv_bfloat16>(fmap, b, n, c, h, w, frames, num_frames, workspace, flags, s);
}

extern "C" int hs2_altcorr_forward_packed(const void* packed1, const void* packed2, int dtype, int b, int n1, int n2,
                                          int c, int h, int w, int h2, int w2, const float* coords,
                                          const int64_t* ii, const int64_t* jj, int m, int radius, void* corr,
                                          int32_t* info, hs2_stream_t stream) {
  using namespace hs2;
  int rc = ac_check("altcorr_forward_packed", b, n1, n2, c, h, w, h2, w2, m, radius);
  if (rc) return rc;
  if (dtype != HS2_F16 && dtype != HS2_BF16) {
    set_error("altcorr_forward_packed: float16 or bfloat16 features only (dtype %d)", dtype);
    return HS2_ERR_DTYPE;
  }
  if (m == 0 || b == 0) return HS2_OK;
  if ((rc = bind_device(corr))) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == HS2_F16)
    return ac_fwd_packed<__half>(packed1, packed2, b, n1, n2, c, h, w, h2, w2, coords, ii, jj, m, radius, corr, info,
                                 s);
  return ac_fwd_packed<__nv_bfloat16>(packed1, packed2, b, n1, n2, c, h, w, h2, w2, coords, ii, jj, m, radius, corr,
                                      info, s);
}

extern "C" int hs2_altcorr_forward(const void* fmap1, const void* fmap2, int dtype, int b, int n1, int n2,
                                   int c, int h, int w, int h2, int w2, const float* coords, const int64_t* ii,
                                   const int64_t* jj, int m, int radius, void* corr, int32_t* info,
                                   hs2_stream_t stream) {
  using namespace hs2;
  int rc = ac_check("altcorr_forward", b, n1, n2, c, h, w, h2, w2, m, radius);
  if (rc) return rc;
  if (m == 0 || b == 0) return HS2_OK;
  if ((rc = bind_device(corr))) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  switch (dtype) {
    case HS2_F32: return ac_fwd<float>(fmap1, fmap2, b, n1, n2, c, h, w, h2, w2, coords, ii, jj, m, radius, corr, info, s);
    case HS2_F16: return ac_fwd<__half>(fmap1, fmap2, b, n1, n2, c, h, w, h2, w2, coords, ii, jj, m, radius, corr, info, s);
    case HS2_BF16:
      return ac_fwd<__nv_bfloat16>(fmap1, fmap2, b, n1, n2, c, h, w, h2, w2, coords, ii, jj, m, radius, corr, info, s);
    case HS2_F64: return ac_fwd<double>(fmap1, fmap2, b, n1, n2, c, h, w, h2, w2, coords, ii, jj, m, radius, corr, info, s);
  }
  set_error("altcorr_forward: unsupported dtype %d", dtype);
  return HS2_ERR_DTYPE;
}

extern "C" int hs2_altcorr_backward_workspace_size(int dtype, int b, int n1, int n2, int c, int h, int w,
                                                   int h2, int w2, size_t* bytes) {
  using namespace hs2;
  if (!bytes) return HS2_ERR_INVALID;
  if (dtype == HS2_F32) {
    *bytes = 0;
    return HS2_OK;
  }
  *bytes = ((size_t)b * n1 * c * h * w + (size_t)b * n2 * c * h2 * w2) * sizeof(float);
  return HS2_OK;
}

extern "C" int hs2_altcorr_backward(const void* fmap1, const void* fmap2, int dtype, int b, int n1, int n2,
                                    int c, int h, int w, int h2, int w2, const float* coords,
                                    const int64_t* ii, const int64_t* jj, int m, const float* grad,
                                    int radius, float scale, void* fmap1_grad, void* fmap2_grad,
                                    int32_t* info, void* workspace, size_t workspace_bytes,
                                    hs2_stream_t stream) {
  using namespace hs2;
  int rc = ac_check("altcorr_backward", b, n1, n2, c, h, w, h2, w2, m, radius);
  if (rc) return rc;
  size_t need = 0;
  hs2_altcorr_backward_workspace_size(dtype, b, n1, n2, c, h, w, h2, w2, &need);
  if (need > 0 && (workspace == nullptr || workspace_bytes < need)) {
    set_error("altcorr_backward: workspace of %zu bytes required", need);
    return HS2_ERR_WORKSPACE;
  }
  if ((rc = bind_device(fmap1_grad))) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  switch (dtype) {
    case HS2_F32:
      return ac_bwd<float>(fmap1, fmap2, b, n1, n2, c, h, w, h2, w2, coords, ii, jj, m, grad, radius, scale,
                           fmap1_grad, fmap2_grad, info, workspace, s);
    case HS2_F16:
      return ac_bwd<__half>(fmap1, fmap2, b, n1, n2, c, h, w, h2, w2, coords, ii, jj, m, grad, radius, scale,
                            fmap1_grad, fmap2_grad, info, workspace, s);
    case HS2_BF16:
      return ac_bwd<__nv_bfloat16>(fmap1, fmap2, b, n1, n2, c, h, w, h2, w2, coords, ii, jj, m, grad, radius,
                                   scale, fmap1_grad, fmap2_grad, info, workspace, s);
  }
  set_error("altcorr_backward: unsupported dtype %d (f32, f16, bf16)", dtype);
  return HS2_ERR_DTYPE;
}

extern "C" int hs2_corr_reproject_lookup_packed(const float* poses, int64_t num_poses, const float* disps,
                                                int64_t num_disps, const float* intrinsics,
                                                const void* const* packed_levels, int levels, int dtype,
                                                int64_t num_frames, int channels, int ht, int wd, const int64_t* ii,
                                                const int64_t* jj, int64_t num_edges, int radius, void* corr,
                                                float* coords1, int32_t* info, hs2_stream_t stream) {
  using namespace hs2;
  if (levels < 1 || levels > 4 || radius < 0 || radius > 8 || channels != 128 || ht <= 0 || wd <= 0 ||
      num_edges < 0 || num_edges > 65535 || num_frames <= 0 || num_frames > (1 << 30) ||
      (ht >> (levels - 1)) <= 0 || (wd >> (levels - 1)) <= 0) {
    set_error("corr_reproject_lookup_packed: bad sizes (levels=%d r=%d C=%d ht=%d wd=%d E=%lld K=%lld); "
              "128 channels and radius <= 8 required", levels, radius, channels, ht, wd, (long long)num_edges,
              (long long)num_frames);
    return HS2_ERR_INVALID;
  }
  if (dtype != HS2_F16 && dtype != HS2_BF16) {
    set_error("corr_reproject_lookup_packed: float16 or bfloat16 features only (dtype %d)", dtype);
    return HS2_ERR_DTYPE;
  }
  if (num_edges == 0) return HS2_OK;
  if (!poses || !disps || !intrinsics || !packed_levels || !ii || !jj || !corr || !info) {
    set_error("corr_reproject_lookup_packed: null pointer argument");
    return HS2_ERR_INVALID;
  }
  AtArgs a{};
  for (int l = 0; l < levels; ++l) {
    if (!packed_levels[l]) {
      set_error("corr_reproject_lookup_packed: feature level %d missing", l);
      return HS2_ERR_INVALID;
    }
    a.p2[l] = packed_levels[l];
  }
  a.p1 = packed_levels[0];
  a.ii = ii;
  a.jj = jj;
  a.corr = corr;
  a.N1 = a.N2 = (int)num_frames;
  a.H = ht, a.W = wd, a.M = (int)num_edges, a.r = radius, a.levels = levels;
  a.info = info;
  a.poses = poses;
  a.disps = disps;
  a.intr = intrinsics;
  a.num_poses = num_poses;
  a.num_disps = num_disps;
  a.coords_out = coords1;
  int rc;
  if ((rc = bind_device(corr))) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  const int ntiles = ((wd + kAtSide - 1) / kAtSide) * ((ht + kAtSide - 1) / kAtSide);
  dim3 grid(ntiles, (unsigned)num_edges, levels);
  HS2_PROF("corr_fused_tile", s);
  if (dtype == HS2_F16) {
    if ((rc = at_prepare<__half, true>())) return rc;
    altcorr_fwd_tile_kernel<__half, true><<<grid, kAtThreads, kAtSmem, s>>>(a);
  } else {
    if ((rc = at_prepare<__nv_bfloat16, true>())) return rc;
    altcorr_fwd_tile_kernel<__nv_bfloat16, true><<<grid, kAtThreads, kAtSmem, s>>>(a);
  }
  HS2_LAUNCH_CHECK("altcorr_fwd_tile_kernel (fused)");
  return HS2_OK;
}
