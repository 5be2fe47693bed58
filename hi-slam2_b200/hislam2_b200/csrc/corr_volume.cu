// All-pairs correlation volume and its 4-level pooling pyramid on the tensor cores.
//
// Replaces the caller-side construction of HI-SLAM2's CorrBlock
// (hislam2/modules/corr.py:29-38 and :63-71):
//   corr[e, y1, x1, y2, x2] = sum_c (fmap1[e, c, y1, x1] / 4) (fmap2[e, c, y2, x2] / 4)
//   level 0 = corr (layout [E, H, W, H, W]),
//   level l = avg_pool2d(level l-1, 2, stride 2) over (y2, x2) (floor sizes),
// i.e. torch.matmul((f1/4)^T, f2/4) followed by three avg_pool2d calls, with the
// same rounding: every level is rounded to the volume's type and pooled from the
// rounded values of the level above, summing the 2x2 window in float in the order
// (y,x), (y,x+1), (y+1,x), (y+1,x+1) and dividing by 4.
//
// Two kernels:
//   corr_pack      fmaps [K, 128, H, W] -> K-major operand rows [K, H*W, 128]
//                  (x 0.25, which is exact; or, for the FP8 form, e4m3 values with one
//                  scale per pixel: q = e4m3(f/4 / s), s = max_c |f/4| / 448);
//   corr_volume    persistent (one CTA per SM), one work unit = (edge, 128 source
//                  pixels).  Warp 0 streams the unit's A tile (128 source pixels x
//                  128 channels) and, per N tile, the B tile of TWO target image
//                  rows (each a box of RW = round_up(W, 16) pixels; pixels past the
//                  frame read as zero) with 3-D TMA boxes (128B swizzle) into a
//                  2-stage ring; warp 1 issues tcgen05.mma (kind::f16 for F16/BF16,
//                  kind::f8f6f4 for E4M3; M = 128, N = 2 RW, accumulator F32) into
//                  one of two 256-column TMEM buffers; warps 2-17 (four per TMEM
//                  lane quarter, each half an image row of the tile) drain the
//                  accumulator (tcgen05.ld), round to the volume type into a
//                  shared staging tile, write level 0 in 16-byte chunks aligned in
//                  global memory, pool level 1 from the two rows of the tile, and
//                  levels 2 and 3 from two-row rings of the levels above.
// The volume is never re-read: the HBM traffic is the pyramid's writes plus the
// operand reads (L2-resident: one frame's operand rows are 848 KB at 43x77).
//
// Limits: 128 channels, W <= 96, H*W < 2^31 / 128.  Output element offsets are 64-bit.
#include <cuda_fp8.h>

#include "profile.cuh"
#include "tc.cuh"

namespace hs2 {

namespace {

constexpr int kCvC = 128;          // feature channels (K of the contraction)
constexpr int kCvMaxW = 96;        // widest image row a B box holds
constexpr int kCvMaxRW = 96;       // round_up(kCvMaxW, 16): accumulator columns per image row
constexpr int kCvEpiWarps = 16;    // four per TMEM lane quarter
constexpr int kCvThreads = 32 * (2 + kCvEpiWarps);   // TMA, MMA, epilogue
constexpr int kCvEpiThreads = 32 * kCvEpiWarps;
constexpr int kCvRowsPerWarp = 128 / kCvEpiWarps;   // staging rows of a warp in phase B
constexpr int kCvStages = 2;
constexpr int kCvTmemCols = 512;   // two 256-column accumulators
constexpr uint32_t kCvASub = 128 * 128;   // one 128-row x 128-byte swizzled sub-tile

// operand forms: F16 / BF16 (kind::f16), E4M3 with per-pixel scales (kind::f8f6f4)
constexpr int kF16 = 0, kBF16 = 1, kE4M3 = 2;
template <int P> struct Prec;
template <> struct Prec<kF16> {
  static constexpr int kEsize = 2, kSub = 2, kFmt = 0;
};
template <> struct Prec<kBF16> {
  static constexpr int kEsize = 2, kSub = 2, kFmt = 1;
};
template <> struct Prec<kE4M3> {
  static constexpr int kEsize = 1, kSub = 1, kFmt = 0;
};

struct CvGeom {
  int H, W, HW, RW, SST;           // grid, row box, staging row stride (elements)
  int H1, W1, H2, W2, H3, W3;      // pooled level sizes
  int levels, mtiles, ntiles;
  int64_t E;
  uint32_t sub_b;                  // bytes of one B sub-tile (2 RW rows x 128 B)
  uint32_t off_b, off_stg, off_r1, off_r2, off_bar, smem;
};

CvGeom cv_geom(int H, int W, int64_t E, int levels, int esub) {
  CvGeom g;
  g.H = H;
  g.W = W;
  g.HW = H * W;
  g.RW = (W + 15) & ~15;
  g.SST = 2 * g.RW + 2;                 // >= 2 W; SST / 2 odd
  g.H1 = H / 2, g.W1 = W / 2, g.H2 = g.H1 / 2, g.W2 = g.W1 / 2, g.H3 = g.H2 / 2, g.W3 = g.W2 / 2;
  g.levels = levels;
  g.mtiles = (g.HW + 127) / 128;
  g.ntiles = (H + 1) / 2;
  g.E = E;
  g.sub_b = (uint32_t)(2 * g.RW * 128);
  const uint32_t a_bytes = 2 * kCvASub;
  g.off_b = a_bytes;
  g.off_stg = g.off_b + kCvStages * esub * g.sub_b;
  g.off_r1 = g.off_stg + 128u * g.SST * 2;
  g.off_r2 = g.off_r1 + 2u * 128 * (g.RW / 2) * 2;
  g.off_bar = (g.off_r2 + 2u * 128 * (g.RW / 4) * 2 + 15) & ~15u;
  g.smem = g.off_bar + 256 + 1024;   // barriers, flags, TMEM slot; 1 KB alignment slack
  return g;
}

template <typename T> __device__ __forceinline__ uint16_t bits16(T v);
template <> __device__ __forceinline__ uint16_t bits16<__half>(__half v) { return __half_as_ushort(v); }
template <> __device__ __forceinline__ uint16_t bits16<__nv_bfloat16>(__nv_bfloat16 v) {
  return __bfloat16_as_ushort(v);
}
template <typename T> __device__ __forceinline__ T from_bits16(uint16_t b);
template <> __device__ __forceinline__ __half from_bits16<__half>(uint16_t b) { return __ushort_as_half(b); }
template <> __device__ __forceinline__ __nv_bfloat16 from_bits16<__nv_bfloat16>(uint16_t b) {
  return __ushort_as_bfloat16(b);
}

__device__ __forceinline__ void epi_sync() { asm volatile("bar.sync 1, %0;" ::"n"(kCvEpiThreads) : "memory"); }
// Barrier of the epilogue warps that also ANDs a predicate over them (a CTA-uniform decision).
__device__ __forceinline__ bool epi_sync_and(bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.and.pred q, 1, %2, p;\n\tselp.u32 %0, 1, 0, q;\n\t}"
      : "=r"(r) : "r"((uint32_t)v), "n"(kCvEpiThreads) : "memory");
  return r != 0;
}
// Bounded wait that ignores the abort flag: used on the way out to let copies and
// MMAs that were already issued land before the CTA releases its memory.
__device__ __forceinline__ void drain_wait(uint32_t bar, uint32_t parity) {
  for (unsigned i = 0; i < tc::kSpin && !tc::mbar_test(bar, parity); ++i) {
  }
}

// Rounded 2x2 average of four 16-bit values, in avg_pool2d's order.
template <typename T>
__device__ __forceinline__ uint16_t pool4(uint16_t a, uint16_t b, uint16_t c, uint16_t d) {
  float s = 0.f;
  s += to_f<T>(from_bits16<T>(a));
  s += to_f<T>(from_bits16<T>(b));
  s += to_f<T>(from_bits16<T>(c));
  s += to_f<T>(from_bits16<T>(d));
  return bits16<T>(from_f<T>(s / 4.0f));
}

}  // namespace

// ----------------------------------------------------------------- pack ---
// fmaps [K, 128, HW] (T) -> rows [K, HW, 128] of the operand type; 64 pixels per CTA.
template <typename T, int P>
__global__ void __launch_bounds__(256) corr_pack_kernel(const T* __restrict__ f, int HW, void* __restrict__ rows,
                                                        float* __restrict__ scale) {
  __shared__ float tile[kCvC][65];
  __shared__ float amax[64];
  const int k = blockIdx.y;
  const int p0 = blockIdx.x * 64;
  const T* src = f + (int64_t)k * kCvC * HW;
  for (int i = threadIdx.x; i < kCvC * 64; i += 256) {
    const int c = i >> 6, p = i & 63;
    tile[c][p] = (p0 + p < HW) ? to_f<T>(src[(int64_t)c * HW + p0 + p]) * 0.25f : 0.f;
  }
  __syncthreads();
  if (P == kE4M3) {
    // per-pixel scale: 8 threads per pixel reduce |x| over the 128 channels
    const int p = threadIdx.x >> 2, part = threadIdx.x & 3;
    float m = 0.f;
    for (int c = part; c < kCvC; c += 4) m = fmaxf(m, fabsf(tile[c][p]));
    m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, 1));
    m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, 2));
    if (part == 0) {
      const float s = m > 0.f ? m / 448.0f : 1.0f;
      amax[p] = s;
      if (p0 + p < HW) scale[(int64_t)k * HW + p0 + p] = s;
    }
    __syncthreads();
    uint8_t* out = static_cast<uint8_t*>(rows) + ((int64_t)k * HW + p0) * kCvC;
    for (int i = threadIdx.x; i < 64 * kCvC / 2; i += 256) {
      const int p = i / (kCvC / 2), c = (i - p * (kCvC / 2)) * 2;
      if (p0 + p >= HW) continue;
      const float inv = 1.0f / amax[p];
      const __nv_fp8x2_storage_t q =
          __nv_cvt_float2_to_fp8x2(make_float2(tile[c][p] * inv, tile[c + 1][p] * inv), __NV_SATFINITE, __NV_E4M3);
      *reinterpret_cast<__nv_fp8x2_storage_t*>(out + (int64_t)p * kCvC + c) = q;
    }
  } else {
    using OpT = typename std::conditional<P == kBF16, __nv_bfloat16, __half>::type;
    OpT* out = static_cast<OpT*>(rows) + ((int64_t)k * HW + p0) * kCvC;
    for (int i = threadIdx.x; i < 64 * kCvC / 2; i += 256) {
      const int p = i / (kCvC / 2), c = (i - p * (kCvC / 2)) * 2;
      if (p0 + p >= HW) continue;
      const uint32_t lo = bits16<OpT>(from_f<OpT>(tile[c][p])), hi = bits16<OpT>(from_f<OpT>(tile[c + 1][p]));
      *reinterpret_cast<uint32_t*>(out + (int64_t)p * kCvC + c) = lo | (hi << 16);
    }
  }
}

// --------------------------------------------------------------- volume ---
struct CvOut {
  uint16_t* lvl[4];
};

template <int P, typename T>
__global__ void __launch_bounds__(kCvThreads, 1)
corr_volume_kernel(const __grid_constant__ CUtensorMap amap, const __grid_constant__ CUtensorMap bmap,
                   const int64_t* __restrict__ ii, const int64_t* __restrict__ jj, int64_t K1, int64_t K2,
                   const float* __restrict__ s1, const float* __restrict__ s2, CvGeom g, CvOut out,
                   int32_t* __restrict__ info) {
  using PR = Prec<P>;
  extern __shared__ uint8_t cv_raw[];
  const uint32_t raw = tc::smem_u32(cv_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  uint8_t* gb = cv_raw + (base - raw);
  uint64_t* bars = reinterpret_cast<uint64_t*>(gb + g.off_bar);
  // a_full, a_empty, b_full[2], b_empty[2], t_full[2], t_empty[2], mma_done
  const uint32_t bar0 = tc::smem_u32(bars);
  const uint32_t a_full = bar0, a_empty = bar0 + 8;
  const uint32_t b_full = bar0 + 16, b_empty = bar0 + 32, t_full = bar0 + 48, t_empty = bar0 + 64;
  const uint32_t mma_done = bar0 + 80;
  volatile int* abort_flag = reinterpret_cast<volatile int*>(gb + g.off_bar + 96);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(gb + g.off_bar + 104);
  uint16_t* stg = reinterpret_cast<uint16_t*>(gb + g.off_stg);
  uint16_t* ring1 = reinterpret_cast<uint16_t*>(gb + g.off_r1);
  uint16_t* ring2 = reinterpret_cast<uint16_t*>(gb + g.off_r2);
  const int R1 = g.RW / 2, R2 = g.RW / 4;   // ring row strides (elements)

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    tc::mbar_init(a_full, 1);
    tc::mbar_init(a_empty, 1);
    for (int s = 0; s < kCvStages; ++s) {
      tc::mbar_init(b_full + 8 * s, 1);
      tc::mbar_init(b_empty + 8 * s, 1);
    }
    for (int b = 0; b < 2; ++b) {
      tc::mbar_init(t_full + 8 * b, 1);
      tc::mbar_init(t_empty + 8 * b, kCvEpiWarps);
    }
    tc::mbar_init(mma_done, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc::smem_u32(tmem_slot)),
                 "r"(kCvTmemCols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = *tmem_slot;

  const int64_t units = g.E * g.mtiles;
  const uint32_t b_stage = (uint32_t)PR::kSub * g.sub_b;
  const int kbox = 128 / PR::kEsize;                  // elements per 128-byte box row

  if (warp == 0) {
    // ------------------------------------------------------------- TMA producer
    if (lane == 0) {
      uint32_t gt = 0, ul = 0;
      for (int64_t u = blockIdx.x; u < units; u += gridDim.x) {
        const int64_t e = u / g.mtiles;
        const int m0 = (int)(u - e * g.mtiles) * 128;
        const int64_t fi = ii[e], fj = jj[e];
        if (fi < 0 || fi >= K1 || fj < 0 || fj >= K2) continue;   // every role skips the unit
        if (ul > 0 && !tc::mbar_wait(a_empty, (ul - 1) & 1, abort_flag)) break;
        ++ul;
        tc::mbar_arrive_tx(a_full, PR::kSub * kCvASub);
        for (int kb = 0; kb < PR::kSub; ++kb)
          tc::tma_load_3d(base + kb * kCvASub, &amap, kb * kbox, m0, (int)fi, a_full);
        bool ok = true;
        for (int j = 0; j < g.ntiles; ++j, ++gt) {
          const int s = gt % kCvStages;
          if (gt >= kCvStages && !tc::mbar_wait(b_empty + 8 * s, ((gt / kCvStages) - 1) & 1, abort_flag)) {
            ok = false;
            break;
          }
          const int nrow = (2 * j + 1 < g.H) ? 2 : 1;
          tc::mbar_arrive_tx(b_full + 8 * s, (uint32_t)(nrow * PR::kSub * g.RW * 128));
          const uint32_t dst = base + g.off_b + s * b_stage;
          for (int r = 0; r < nrow; ++r)
            for (int kb = 0; kb < PR::kSub; ++kb)
              tc::tma_load_3d(dst + kb * g.sub_b + r * g.RW * 128, &bmap, kb * kbox, (2 * j + r) * g.W, (int)fj,
                              b_full + 8 * s);
        }
        if (!ok) break;
      }
      // let the copies already issued land before the CTA's shared memory is released
      if (ul > 0) drain_wait(a_full, (ul - 1) & 1);
      for (uint32_t k = gt > kCvStages ? gt - kCvStages : 0; k < gt; ++k)
        drain_wait(b_full + 8 * (k % kCvStages), (k / kCvStages) & 1);
    }
  } else if (warp == 1) {
    // ------------------------------------------------------------- MMA issuer
    if (lane == 0) {
      uint32_t gt = 0, ul = 0;
      for (int64_t u = blockIdx.x; u < units; u += gridDim.x) {
        const int64_t e = u / g.mtiles;
        const int64_t fi = ii[e], fj = jj[e];
        if (fi < 0 || fi >= K1 || fj < 0 || fj >= K2) continue;
        if (!tc::mbar_wait(a_full, ul & 1, abort_flag)) break;
        ++ul;
        bool ok = true;
        for (int j = 0; j < g.ntiles; ++j, ++gt) {
          const int s = gt % kCvStages, b = gt & 1;
          if (!tc::mbar_wait(b_full + 8 * s, (gt / kCvStages) & 1, abort_flag) ||
              (gt >= 2 && !tc::mbar_wait(t_empty + 8 * b, ((gt >> 1) - 1) & 1, abort_flag))) {
            ok = false;
            break;
          }
          tc::fence_after();
          const int nrow = (2 * j + 1 < g.H) ? 2 : 1;
          const uint32_t id = tc::idesc(128, nrow * g.RW, PR::kFmt);
          const uint32_t bsrc = base + g.off_b + s * b_stage;
          const uint32_t d = tmem + (uint32_t)(b * 256);
#pragma unroll
          for (int kb = 0; kb < PR::kSub; ++kb)
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) {
              const uint64_t ad = tc::desc_sw128(base + kb * kCvASub + kk * 32);
              const uint64_t bd = tc::desc_sw128(bsrc + kb * g.sub_b + kk * 32);
              if (P == kE4M3) tc::mma_f8(d, ad, bd, id, (kb | kk) ? 1u : 0u);
              else tc::mma_f16(d, ad, bd, id, (kb | kk) ? 1u : 0u);
            }
          tc::commit(b_empty + 8 * s);
          tc::commit(t_full + 8 * b);
        }
        if (!ok) break;
        tc::commit(a_empty);
      }
      // every MMA issued has completed before TMEM is released
      tc::commit(mma_done);
      drain_wait(mma_done, 0);
    }
  } else {
    // ------------------------------------------------------------- epilogue
    // Phase A (per tile): warp (quarter q, half h) reads its 32 accumulator rows' columns
    // of image row h from TMEM, rounds them and stores them, 4 bytes at a time, into the
    // staging row of each source pixel: segment layout, image row 0 at [0, W), row 1 at
    // [W, 2W) (row stride SST, SST/2 odd: the 32 rows of a store hit 32 banks).
    // Phase B: warp ew owns staging rows 16 ew .. 16 ew + 15.  Level 0: the row's
    // segment is one contiguous run of the volume row; it is written in 16-byte chunks
    // aligned in GLOBAL memory (lane = (row, chunk parity)), each gathered from 8 staged
    // elements -- whole sectors per store; the two chunks that straddle the segment's
    // ends go element by element.  Levels 1-3: lanes over x per row, each pooled value
    // written to its ring and to global memory by the lane that forms it.
    const int ew = warp - 2;                 // 0..15
    const int q = warp & 3;                  // TMEM lane quarter
    const int h = (ew >> 2) >> 1;            // image row of the tile (phase A)
    const int half = (ew >> 2) & 1;          // which half of the row's RW columns
    const int hw = g.RW / 2;                 // columns per warp (a multiple of 8)
    const int r = q * 32 + lane;             // accumulator row = source pixel within the unit
    const int pa = lane % kCvRowsPerWarp, pb = lane / kCvRowsPerWarp;
    const int prow = kCvRowsPerWarp * ew + pa;   // phase B staging row of this lane
    constexpr int kChunkLanes = 32 / kCvRowsPerWarp;
    const int64_t L1n = (int64_t)g.H1 * g.W1, L2n = (int64_t)g.H2 * g.W2, L3n = (int64_t)g.H3 * g.W3;
    uint32_t gt = 0;
    for (int64_t u = blockIdx.x; u < units; u += gridDim.x) {
      const int64_t e = u / g.mtiles;
      const int m0 = (int)(u - e * g.mtiles) * 128;
      const int64_t fi = ii[e], fj = jj[e];
      if (fi < 0 || fi >= K1 || fj < 0 || fj >= K2) {
        if (tid == 64 && m0 == 0) atomicOr(info, HS2_DEV_BAD_INDEX);
        continue;
      }
      float sa = 1.f;
      if (P == kE4M3) sa = (m0 + r < g.HW) ? s1[fi * g.HW + m0 + r] : 0.f;
      bool ok = true;
      for (int j = 0; j < g.ntiles; ++j, ++gt) {
        const int b = gt & 1;
        const int nrow = (2 * j + 1 < g.H) ? 2 : 1;
        ok = tc::mbar_wait(t_full + 8 * b, (gt >> 1) & 1, abort_flag);
        tc::fence_after();
        if (ok && h < nrow) {
          constexpr int kHalf = kCvMaxRW / 2;
          uint32_t v[kHalf];
#pragma unroll
          for (int c0 = 0; c0 < kHalf; c0 += 8) {
            if (c0 < hw) {
              uint32_t t8[8];
              tc::ld8(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * 256 + h * g.RW + half * hw + c0), t8);
#pragma unroll
              for (int k = 0; k < 8; ++k) v[c0 + k] = t8[k];
            }
          }
          tc::ld_wait();
          const int xb = half * hw;          // first image column of this warp
          if (P == kE4M3) {
            // column scales of the warp's columns (lane c holds columns xb + c, xb + c + 32)
            float sc[(kHalf + 31) / 32];
#pragma unroll
            for (int k = 0; k < (kHalf + 31) / 32; ++k) {
              const int x = xb + lane + 32 * k;
              sc[k] = (lane + 32 * k < hw && x < g.W) ? s2[fj * g.HW + (int64_t)(2 * j + h) * g.W + x] : 0.f;
            }
#pragma unroll
            for (int x = 0; x < kHalf; ++x) {
              const float scale = __shfl_sync(0xffffffffu, sc[x >> 5], x & 31);
              v[x] = __float_as_uint(__uint_as_float(v[x]) * sa * scale);
            }
          }
          uint16_t* srow = stg + r * g.SST + h * g.W + xb;
          const int nv = min(hw, g.W - xb);   // valid columns of this warp
          auto q16 = [&](int x) -> uint32_t { return (uint32_t)bits16<T>(from_f<T>(__uint_as_float(v[x]))); };
          if (((h * g.W + xb) & 1) == 0) {
#pragma unroll
            for (int x = 0; x < kHalf; x += 2) {
              if (x + 1 < nv) *reinterpret_cast<uint32_t*>(srow + x) = q16(x) | (q16(x + 1) << 16);
              else if (x < nv) srow[x] = (uint16_t)q16(x);
            }
          } else {
            if (nv > 0) srow[0] = (uint16_t)q16(0);
#pragma unroll
            for (int x = 1; x < kHalf; x += 2) {
              if (x + 1 < nv) *reinterpret_cast<uint32_t*>(srow + x) = q16(x) | (q16(x + 1) << 16);
              else if (x < nv) srow[x] = (uint16_t)q16(x);
            }
          }
        }
        tc::fence_before();
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(t_empty + 8 * b);
        ok = epi_sync_and(ok);               // uniform over the epilogue warps from here on
        if (ok) {
          // ---- level 0: global-aligned 16-byte chunks of this lane's row
          const int nseg = nrow * g.W;
          {
            const int m = m0 + prow;
            if (m < g.HW) {
              const int64_t G0 = (e * g.HW + m) * (int64_t)g.HW + (int64_t)(2 * j) * g.W;
              const int off = (int)(G0 & 7);
              const int nch = (off + nseg + 7) >> 3;
              uint16_t* gb0 = out.lvl[0] + (G0 - off);
              const uint16_t* sr = stg + prow * g.SST;
              for (int k = pb; k < nch; k += kChunkLanes) {
                const int c0 = 8 * k - off;
                if (c0 >= 0 && c0 + 8 <= nseg) {
                  uint32_t wv[4];
#pragma unroll
                  for (int i = 0; i < 4; ++i) wv[i] = (uint32_t)sr[c0 + 2 * i] | ((uint32_t)sr[c0 + 2 * i + 1] << 16);
                  *reinterpret_cast<uint4*>(gb0 + 8 * k) = make_uint4(wv[0], wv[1], wv[2], wv[3]);
                } else {
#pragma unroll
                  for (int i = 0; i < 8; ++i) {
                    const int c = c0 + i;
                    if (c >= 0 && c < nseg) gb0[8 * k + i] = sr[c];
                  }
                }
              }
            }
          }
          // ---- levels 1-3: rows 16 ew .. 16 ew + 15, lanes over x
          if (g.levels > 1 && j < g.H1) {
            uint16_t* r1 = ring1 + (j & 1) * 128 * R1;
            const int rbase = kCvRowsPerWarp * ew;
            // items (row, x) of the warp's rows, lane-strided, stepped without division
            int a2 = 0, x = lane;
            while (x >= g.W1) { x -= g.W1; ++a2; }
            for (; a2 < kCvRowsPerWarp;) {
              const int rr = rbase + a2;
              const uint16_t* sr = stg + rr * g.SST;
              const uint16_t pv = pool4<T>(sr[2 * x], sr[2 * x + 1], sr[g.W + 2 * x], sr[g.W + 2 * x + 1]);
              r1[rr * R1 + x] = pv;
              if (m0 + rr < g.HW) out.lvl[1][(e * g.HW + m0 + rr) * L1n + (int64_t)j * g.W1 + x] = pv;
              x += 32;
              while (x >= g.W1) { x -= g.W1; ++a2; }
            }
            __syncwarp();
            const int j2 = j >> 1;
            if (g.levels > 2 && (j & 1) && j2 < g.H2) {
              uint16_t* r2 = ring2 + (j2 & 1) * 128 * R2;
              a2 = 0;
              x = lane;
              while (x >= g.W2) { x -= g.W2; ++a2; }
              for (; a2 < kCvRowsPerWarp;) {
                const int rr = rbase + a2;
                const uint16_t* p0 = ring1 + rr * R1;              // level-1 row j-1 (slot 0)
                const uint16_t* p1 = ring1 + 128 * R1 + rr * R1;   // level-1 row j (slot 1)
                const uint16_t pv = pool4<T>(p0[2 * x], p0[2 * x + 1], p1[2 * x], p1[2 * x + 1]);
                r2[rr * R2 + x] = pv;
                if (m0 + rr < g.HW) out.lvl[2][(e * g.HW + m0 + rr) * L2n + (int64_t)j2 * g.W2 + x] = pv;
                x += 32;
                while (x >= g.W2) { x -= g.W2; ++a2; }
              }
              __syncwarp();
              const int j3 = j2 >> 1;
              if (g.levels > 3 && (j2 & 1) && j3 < g.H3) {
                a2 = 0;
                x = lane;
                while (x >= g.W3) { x -= g.W3; ++a2; }
                for (; a2 < kCvRowsPerWarp;) {
                  const int rr = rbase + a2;
                  const uint16_t* p0 = ring2 + rr * R2;
                  const uint16_t* p1 = ring2 + 128 * R2 + rr * R2;
                  const uint16_t pv = pool4<T>(p0[2 * x], p0[2 * x + 1], p1[2 * x], p1[2 * x + 1]);
                  if (m0 + rr < g.HW) out.lvl[3][(e * g.HW + m0 + rr) * L3n + (int64_t)j3 * g.W3 + x] = pv;
                  x += 32;
                  while (x >= g.W3) { x -= g.W3; ++a2; }
                }
              }
            }
          }
        }
        epi_sync();                          // the staging tile is rewritten by the next tile
        if (!ok) break;
      }
      if (!ok) break;
    }
  }
  if (*abort_flag && tid == 0) atomicOr(info, HS2_DEV_TIMEOUT);
  tc::fence_before();
  __syncthreads();
  if (warp == 1) {
    tc::fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCvTmemCols) : "memory");
  }
}

// ------------------------------------------------------------------- host ---
namespace {

int cv_check(int64_t E, int64_t K1, int64_t K2, int C, int H, int W, int dtype, int precision, int levels) {
  if (E < 0 || K1 < 0 || K2 < 0 || H <= 0 || W <= 0 || levels < 1 || levels > 4) {
    set_error("corr_volume: bad sizes E=%lld K1=%lld K2=%lld H=%d W=%d levels=%d", (long long)E, (long long)K1,
              (long long)K2, H, W, levels);
    return HS2_ERR_INVALID;
  }
  if (C != kCvC) {
    set_error("corr_volume: %d feature channels (the kernel contracts exactly 128)", C);
    return HS2_ERR_INVALID;
  }
  if (W > kCvMaxW) {
    set_error("corr_volume: W=%d exceeds %d (one image row per TMA box)", W, kCvMaxW);
    return HS2_ERR_INVALID;
  }
  if ((int64_t)H * W * kCvC >= (int64_t(1) << 31)) {
    set_error("corr_volume: H*W=%lld too large", (long long)H * W);
    return HS2_ERR_INVALID;
  }
  if (dtype != HS2_F16 && dtype != HS2_BF16) {
    set_error("corr_volume: fmaps must be float16 or bfloat16");
    return HS2_ERR_DTYPE;
  }
  if (precision != HS2_CV_NATIVE && precision != HS2_CV_E4M3) {
    set_error("corr_volume: unknown precision %d", precision);
    return HS2_ERR_INVALID;
  }
  return HS2_OK;
}

size_t cv_workspace(int64_t K1, int64_t K2, int H, int W, int precision) {
  const int64_t HW = (int64_t)H * W;
  const int es = precision == HS2_CV_E4M3 ? 1 : 2;
  size_t bytes = (size_t)(K1 + K2) * HW * kCvC * es;
  bytes = (bytes + 255) & ~size_t(255);
  if (precision == HS2_CV_E4M3) bytes += ((size_t)(K1 + K2) * HW * sizeof(float) + 255) & ~size_t(255);
  return bytes;
}

template <typename T, int P>
int cv_pack(const void* f, int64_t K, int HW, void* rows, float* scale, cudaStream_t s) {
  if (K == 0) return HS2_OK;
  dim3 grid((HW + 63) / 64, (unsigned)K);
  HS2_PROF("corr_pack", s);
  corr_pack_kernel<T, P><<<grid, 256, 0, s>>>(static_cast<const T*>(f), HW, rows, scale);
  HS2_LAUNCH_CHECK("corr_pack_kernel");
  return HS2_OK;
}

// Operand rows [K, HW, 128] as a 3-D tensor (channels innermost); a box is 128 bytes of
// channels x box_rows pixels of one frame, so rows past a frame's last pixel read as zero.
int cv_map(CUtensorMap* map, void* rows, int64_t K, int HW, int P, int box_rows) {
  const int esize = P == kE4M3 ? 1 : 2;
  const cuuint64_t dims[3] = {(cuuint64_t)kCvC, (cuuint64_t)HW, (cuuint64_t)K};
  const cuuint64_t strides[2] = {(cuuint64_t)kCvC * esize, (cuuint64_t)HW * kCvC * esize};
  const cuuint32_t box[3] = {(cuuint32_t)(128 / esize), (cuuint32_t)box_rows, 1};
  const CUtensorMapDataType t = P == kE4M3  ? CU_TENSOR_MAP_DATA_TYPE_UINT8
                                : P == kBF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                                             : CU_TENSOR_MAP_DATA_TYPE_FLOAT16;
  return tc::encode_tiled(map, t, 3, rows, dims, strides, box, CU_TENSOR_MAP_SWIZZLE_128B);
}

template <int P, typename T>
int cv_launch(const CvGeom& g, void* rows1, void* rows2, const float* s1, const float* s2, int64_t K1, int64_t K2,
              const int64_t* ii, const int64_t* jj, CvOut out, int32_t* info, cudaStream_t s) {
  CUtensorMap amap, bmap;
  int rc;
  if ((rc = cv_map(&amap, rows1, K1, g.HW, P, 128))) return rc;
  if ((rc = cv_map(&bmap, rows2, K2, g.HW, P, g.RW))) return rc;
  static DeviceOnce once;
  int dev = 0;
  HS2_CUDA(cudaGetDevice(&dev));
  static std::atomic<int> sms[kMaxDevices];
  rc = once.run(dev, [&]() -> int {
    HS2_CUDA(cudaFuncSetAttribute(corr_volume_kernel<P, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  227 * 1024));
    int n = 0;
    HS2_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
    sms[dev].store(n);
    return HS2_OK;
  });
  if (rc) return rc;
  const int64_t units = g.E * g.mtiles;
  if (units == 0) return HS2_OK;
  const int grid = (int)std::min<int64_t>(units, sms[dev].load());
  HS2_PROF("corr_volume", s);
  corr_volume_kernel<P, T><<<grid, kCvThreads, g.smem, s>>>(amap, bmap, ii, jj, K1, K2, s1, s2, g, out, info);
  HS2_LAUNCH_CHECK("corr_volume_kernel");
  return HS2_OK;
}

}  // namespace

}  // namespace hs2

extern "C" int hs2_corr_volume_workspace_size(int64_t k1, int64_t k2, int channels, int ht, int wd, int dtype,
                                              int precision, size_t* bytes) {
  using namespace hs2;
  if (!bytes) {
    set_error("corr_volume_workspace_size: null output");
    return HS2_ERR_INVALID;
  }
  const int rc = cv_check(0, k1, k2, channels, ht, wd, dtype, precision, 4);
  if (rc) return rc;
  *bytes = cv_workspace(k1, k2, ht, wd, precision);
  return HS2_OK;
}

extern "C" int hs2_corr_volume(const void* fmap1, int64_t k1, const void* fmap2, int64_t k2, int channels, int ht,
                               int wd, int dtype, const int64_t* ii, const int64_t* jj, int64_t num_pairs,
                               int precision, int levels, void* const* pyramid, int32_t* info, void* workspace,
                               size_t workspace_bytes, hs2_stream_t stream) {
  using namespace hs2;
  int rc = cv_check(num_pairs, k1, k2, channels, ht, wd, dtype, precision, levels);
  if (rc) return rc;
  if (num_pairs == 0) return HS2_OK;
  if (!fmap1 || !fmap2 || !ii || !jj || !pyramid || !info) {
    set_error("corr_volume: null pointer argument");
    return HS2_ERR_INVALID;
  }
  for (int l = 0; l < levels; ++l) {
    const int hl = ht >> l, wl = wd >> l;
    if (hl > 0 && wl > 0 && !pyramid[l]) {
      set_error("corr_volume: level %d output missing", l);
      return HS2_ERR_INVALID;
    }
  }
  const size_t need = cv_workspace(k1, k2, ht, wd, precision);
  if (!workspace || workspace_bytes < need) {
    set_error("corr_volume: workspace of %zu bytes required", need);
    return HS2_ERR_WORKSPACE;
  }
  if ((rc = bind_device(fmap1))) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  const int HW = ht * wd;
  const int es = precision == HS2_CV_E4M3 ? 1 : 2;
  uint8_t* ws = static_cast<uint8_t*>(workspace);
  void* rows1 = ws;
  void* rows2 = ws + (size_t)k1 * HW * kCvC * es;
  float* sc1 = nullptr;
  float* sc2 = nullptr;
  if (precision == HS2_CV_E4M3) {
    size_t off = ((size_t)(k1 + k2) * HW * kCvC + 255) & ~size_t(255);
    sc1 = reinterpret_cast<float*>(ws + off);
    sc2 = sc1 + (size_t)k1 * HW;
  }
  CvOut out;
  for (int l = 0; l < 4; ++l) out.lvl[l] = l < levels ? static_cast<uint16_t*>(pyramid[l]) : nullptr;
  const CvGeom g = cv_geom(ht, wd, num_pairs, levels, precision == HS2_CV_E4M3 ? 1 : 2);
  if (dtype == HS2_F16) {
    if (precision == HS2_CV_E4M3) {
      if ((rc = cv_pack<__half, kE4M3>(fmap1, k1, HW, rows1, sc1, s))) return rc;
      if ((rc = cv_pack<__half, kE4M3>(fmap2, k2, HW, rows2, sc2, s))) return rc;
      return cv_launch<kE4M3, __half>(g, rows1, rows2, sc1, sc2, k1, k2, ii, jj, out, info, s);
    }
    if ((rc = cv_pack<__half, kF16>(fmap1, k1, HW, rows1, nullptr, s))) return rc;
    if ((rc = cv_pack<__half, kF16>(fmap2, k2, HW, rows2, nullptr, s))) return rc;
    return cv_launch<kF16, __half>(g, rows1, rows2, nullptr, nullptr, k1, k2, ii, jj, out, info, s);
  }
  if (precision == HS2_CV_E4M3) {
    if ((rc = cv_pack<__nv_bfloat16, kE4M3>(fmap1, k1, HW, rows1, sc1, s))) return rc;
    if ((rc = cv_pack<__nv_bfloat16, kE4M3>(fmap2, k2, HW, rows2, sc2, s))) return rc;
    return cv_launch<kE4M3, __nv_bfloat16>(g, rows1, rows2, sc1, sc2, k1, k2, ii, jj, out, info, s);
  }
  if ((rc = cv_pack<__nv_bfloat16, kBF16>(fmap1, k1, HW, rows1, nullptr, s))) return rc;
  if ((rc = cv_pack<__nv_bfloat16, kBF16>(fmap2, k2, HW, rows2, nullptr, s))) return rc;
  return cv_launch<kBF16, __nv_bfloat16>(g, rows1, rows2, nullptr, nullptr, k1, k2, ii, jj, out, info, s);
}
