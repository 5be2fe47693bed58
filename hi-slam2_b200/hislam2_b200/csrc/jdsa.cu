// Mono-prior depth / scale alignment step: HI-SLAM2's JDSA (hislam2/geom/ba.py:170-219 with
// get_prior_depth_aligned :159-167 and geom/chol.py:schur_solve_mono_prior :80-107).
//
// The reference builds the step from dense tensors: the bilinear scale Jacobian [M,H,W,hs,ws],
// E [M*D, M*HW] (D = hs*ws scale unknowns per frame), E Q E^T and one Cholesky of the
// [M*D, M*D] system, then inv(L) E Q for the depth covariance.  Its scatter keys are
// (kx', kx') with kx' = kx - kx[0] (kx = unique(ii)), so H and E only have diagonal blocks:
// the reduced system is block diagonal, one D x D block per source frame, and the whole
// step is per frame.  Block b couples the prior terms of frame kx[0] + b (when that frame
// is a source frame; else none) with row b of C, w, eta and the prior mask (frame kx[b]):
// the two are the same frame whenever kx is contiguous, and this pairing is what the
// reference computes when it is not.
//
//   proj_trans         (geometry.cu) the depth-only Schur terms C, w [M, HW];
//   jdsa_solve         CTA per block b: per pixel, in FP32 as the reference,
//                        Q = 1 / (C + m alpha + (1 - m) eta),  w' = w - m alpha rd,
//                        a = prior [> 0] of the source frame, J = -a (wa, wb, wc, wd) at the
//                        pixel's interpolation cell,
//                      summed in FP64 per cell over the CTA: S += alpha a^2 (1 - alpha Q) w w^T,
//                      diag(H) += alpha a^2 w^2, v += alpha a w (rd_src + Q w'); then
//                      S + diag(0.1 + 1e-4 diag(H)) = L L^T in FP64 by one thread (D <= 16),
//                      dso = S^-1 v; second pass: dz = Q (w' + alpha a (w . dso_cell)),
//                      disps_out = clamp(where(d + dz > 10, 0, d + dz), min = 0.001) and
//                      dzcov = (alpha a Q)^2 w^T S^-1_cell w + Q  (= |L^-1 E Q|^2 + Q).
//                      CTAs M .. M + num_disps - 1 copy the frames that are not source frames
//                      through the same where / clamp (the reference applies both to the
//                      whole window).
//   jdsa_scales        dscales[kx[b]] += dso[b], skipped when a block was not positive
//                      definite or an index was bad (the reference raises before it).
#include "common.cuh"
#include "profile.cuh"

namespace hs2 {

namespace {

constexpr int kJdThreads = 256;
constexpr int kJdWarps = kJdThreads / 32;
constexpr int kJdMaxD = 16;
constexpr int kJdSums = 18;        // one cell: 10 Gram terms, 4 diag(H) terms, 4 rhs terms
constexpr int kJdMaxAxis = 4096;   // ht, wd (the grid axes are staged in shared memory)
constexpr double kJdEp = 0.1;      // schur_solve_mono_prior's ep and lm (chol.py:80)
constexpr double kJdLm = 1e-4;

struct JdArgs {
  const float* disps;
  int64_t num_disps;
  int ht, wd;
  const float* C;
  const float* w;
  const float* eta;
  const float* prior;
  int64_t num_prior;
  const float* dscales;
  int64_t num_scales;
  int hs, ws;
  const float* gy;
  const float* gx;
  const int64_t* kx;
  int M;
  float alpha;
  float* dso;     // [M, D]
  float* out;     // [num_disps, H, W]
  float* dzcov;   // [M, HW] or null
  int32_t* info;
};

__device__ __forceinline__ int find_sorted(const int64_t* kx, int M, int64_t f) {
  int lo = 0, hi = M - 1;
  while (lo <= hi) {
    const int mid = (lo + hi) >> 1;
    const int64_t v = kx[mid];
    if (v == f) return mid;
    if (v < f) lo = mid + 1;
    else hi = mid - 1;
  }
  return -1;
}

// torch.where(d > 10, 0, d).clamp(min=0.001); NaN passes through as in torch
__device__ __forceinline__ float jd_clean(float d) {
  d = d > 10.f ? 0.f : d;
  return d < 0.001f ? 0.001f : d;
}

// One pixel's interpolation cell: bi_inter_kernel's weights (droid_kernels.cu:1297-1306)
// and the D-indices of the corners (y0,x0), (y1,x0), (y0,x1), (y1,x1) they multiply.
struct Cell {
  float wt[4];
  int pos[4];
};

__device__ __forceinline__ Cell make_cell(float x, float y, int cx, int cy, int ws) {
  const float x0 = (float)cx, y0 = (float)cy, x1 = x0 + 1.f, y1 = y0 + 1.f;
  Cell c;
  c.wt[0] = (x1 - x) * (y1 - y);
  c.wt[1] = (x1 - x) * (y - y0);
  c.wt[2] = (x - x0) * (y1 - y);
  c.wt[3] = (x - x0) * (y - y0);
  c.pos[0] = cy * ws + cx;
  c.pos[1] = (cy + 1) * ws + cx;
  c.pos[2] = cy * ws + cx + 1;
  c.pos[3] = (cy + 1) * ws + cx + 1;
  return c;
}

__device__ __forceinline__ float interp(const float* S, const Cell& c) {
  return c.wt[0] * S[c.pos[0]] + c.wt[1] * S[c.pos[1]] + c.wt[2] * S[c.pos[2]] + c.wt[3] * S[c.pos[3]];
}

// Row terms of pixel k of block b (frame fr): Q, w' and the disparity itself.
struct RowTerms {
  float Q, wq, d;
};

__device__ __forceinline__ RowTerms row_terms(const JdArgs& A, int b, int64_t fr, int HW, int k, const float* sc,
                                              const Cell& c) {
  const int64_t rk = (int64_t)b * HW + k, fk = fr * HW + k;
  const float pr = A.prior[fk];
  const float m = pr > 0.f ? 1.f : 0.f;
  const float d = A.disps[fk];
  const float rd = d - pr * interp(sc, c);
  const float Cb = A.C[rk] + m * A.alpha + (1.f - m) * A.eta[rk];
  RowTerms t;
  t.Q = 1.0f / Cb;
  t.wq = A.w[rk] - m * A.alpha * rd;
  t.d = d;
  return t;
}

template <int N>
__device__ __forceinline__ void block_sum(double (&acc)[N], double (*red)[N], double* tot) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < N; ++i) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc[i] += __shfl_down_sync(0xffffffffu, acc[i], off);
  }
  if (lane == 0) {
#pragma unroll
    for (int i = 0; i < N; ++i) red[warp][i] = acc[i];
  }
  __syncthreads();
  if (threadIdx.x < N) {
    double s = 0.0;
    for (int q = 0; q < kJdWarps; ++q) s += red[q][threadIdx.x];
    tot[threadIdx.x] = s;
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kJdThreads)
jdsa_solve_kernel(const JdArgs A) {
  extern __shared__ float jd_axes[];   // gy [ht] then gx [wd]
  __shared__ double red[kJdWarps][kJdSums];
  __shared__ double tot[kJdSums];
  __shared__ double S[kJdMaxD][kJdMaxD + 1];
  __shared__ double Lc[kJdMaxD][kJdMaxD + 1];
  __shared__ double Li[kJdMaxD][kJdMaxD + 1];
  __shared__ double Hd[kJdMaxD], v[kJdMaxD];
  __shared__ float dso[kJdMaxD];
  __shared__ float Si[kJdMaxD][kJdMaxD + 1];
  __shared__ float sc_r[kJdMaxD], sc_s[kJdMaxD];
  __shared__ int bad, failed;
  const int HW = A.ht * A.wd, D = A.hs * A.ws, tid = threadIdx.x;
  const int g = blockIdx.x;
  if (g >= A.M) {
    // a frame of the window that is not a source frame: the where / clamp only
    const int64_t f = g - A.M;
    if (find_sorted(A.kx, A.M, f) >= 0) return;
    const float* src = A.disps + f * HW;
    float* dst = A.out + f * HW;
    for (int k = tid; k < HW; k += kJdThreads) dst[k] = jd_clean(src[k]);
    return;
  }
  const int b = g;
  const int64_t fr = A.kx[b];
  const int ms = find_sorted(A.kx, A.M, A.kx[0] + b);   // source of block b's prior terms
  const int64_t fs = ms >= 0 ? A.kx[ms] : fr;
  if (tid == 0) {
    bad = fr < 0 || fr >= A.num_disps || fr >= A.num_prior || fr >= A.num_scales || (b > 0 && A.kx[b - 1] >= fr) ||
          fs < 0 || fs >= A.num_disps || fs >= A.num_prior || fs >= A.num_scales;
    failed = 0;
  }
  float* gy = jd_axes;
  float* gx = jd_axes + A.ht;
  for (int i = tid; i < A.ht; i += kJdThreads) gy[i] = A.gy[i];
  for (int j = tid; j < A.wd; j += kJdThreads) gx[j] = A.gx[j];
  if (tid < D) {
    sc_r[tid] = A.dscales[fr * D + tid];
    sc_s[tid] = A.dscales[fs * D + tid];
    Hd[tid] = 0.0;
    v[tid] = 0.0;
  }
  for (int e = tid; e < kJdMaxD * kJdMaxD; e += kJdThreads) S[e / kJdMaxD][e % kJdMaxD] = 0.0;
  __syncthreads();
  // every grid coordinate needs its 2x2 cell inside the scale grid (bi_inter's bound)
  for (int i = tid; i < A.ht + A.wd; i += kJdThreads) {
    const float c = floorf(i < A.ht ? gy[i] : gx[i - A.ht]);
    const int n = i < A.ht ? A.hs : A.ws;
    if (!(c >= 0.f && c + 1.f < (float)n)) bad = 1;
  }
  __syncthreads();
  if (bad) {
    if (tid == 0) atomicOr(A.info, HS2_DEV_BAD_INDEX);
    return;
  }
  const bool has_src = ms >= 0;
  const float alpha = A.alpha;

  // ---- pass 1: the block's Schur complement and right-hand side, cell by cell
  for (int cy = 0; cy < A.hs - 1; ++cy) {
    for (int cx = 0; cx < A.ws - 1; ++cx) {
      double acc[kJdSums];
#pragma unroll
      for (int i = 0; i < kJdSums; ++i) acc[i] = 0.0;
      if (has_src) {
        for (int k = tid; k < HW; k += kJdThreads) {
          const int i = k / A.wd, j = k - i * A.wd;
          if ((int)floorf(gy[i]) != cy || (int)floorf(gx[j]) != cx) continue;
          const Cell c = make_cell(gx[j], gy[i], cx, cy, A.ws);
          const RowTerms r = row_terms(A, b, fr, HW, k, sc_r, c);
          const int64_t sk = fs * HW + k;
          const float ps = A.prior[sk];
          const float a = ps > 0.f ? ps : 0.f;
          const float rds = A.disps[sk] - ps * interp(sc_s, c);
          const double ca = (double)(alpha * a * a * (1.0f - alpha * r.Q));
          const double ha = (double)(alpha * a * a);
          const double va = (double)(alpha * a * (rds + r.Q * r.wq));
          int q = 0;
#pragma unroll
          for (int kk = 0; kk < 4; ++kk) {
#pragma unroll
            for (int ll = kk; ll < 4; ++ll) acc[q++] += ca * c.wt[kk] * c.wt[ll];
          }
#pragma unroll
          for (int kk = 0; kk < 4; ++kk) {
            acc[10 + kk] += ha * c.wt[kk] * c.wt[kk];
            acc[14 + kk] += va * c.wt[kk];
          }
        }
      }
      block_sum<kJdSums>(acc, red, tot);
      if (tid < kJdSums) {
        const int p0 = cy * A.ws + cx;
        const int pos[4] = {p0, p0 + A.ws, p0 + 1, p0 + A.ws + 1};
        if (tid < 10) {
          int kk = 0, q = tid;
          while (q >= 4 - kk) { q -= 4 - kk; ++kk; }
          const int ll = kk + q;
          S[pos[kk]][pos[ll]] += tot[tid];
          if (ll != kk) S[pos[ll]][pos[kk]] += tot[tid];
        } else if (tid < 14) {
          Hd[pos[tid - 10]] += tot[tid];
        } else {
          v[pos[tid - 14]] += tot[tid];
        }
      }
      __syncthreads();
    }
  }

  // ---- damped D x D solve in FP64 (one thread; D <= 16)
  if (tid == 0) {
    bool ok = true;
    for (int k = 0; k < D && ok; ++k) {
      for (int l = 0; l <= k; ++l) {
        double s = S[k][l] + (k == l ? kJdEp + kJdLm * Hd[k] : 0.0);
        for (int m = 0; m < l; ++m) s -= Lc[k][m] * Lc[l][m];
        if (l == k) {
          if (!(s > 0.0)) { ok = false; break; }
          Lc[k][k] = sqrt(s);
        } else {
          Lc[k][l] = s / Lc[l][l];
        }
      }
    }
    double y[kJdMaxD];
    if (ok) {
      for (int k = 0; k < D; ++k) {
        double s = v[k];
        for (int m = 0; m < k; ++m) s -= Lc[k][m] * y[m];
        y[k] = s / Lc[k][k];
      }
      for (int k = D - 1; k >= 0; --k) {
        double s = y[k];
        for (int m = k + 1; m < D; ++m) s -= Lc[m][k] * y[m];
        y[k] = s / Lc[k][k];
      }
    }
    for (int k = 0; k < D; ++k) {
      dso[k] = ok ? (float)y[k] : 0.f;
      A.dso[(int64_t)b * D + k] = dso[k];
    }
    if (!ok) {
      failed = 1;
      atomicOr(A.info, HS2_DEV_NOT_PD);
    }
  }
  __syncthreads();
  if (A.dzcov) {
    // columns of L^-1 by forward substitution (thread k: L x = e_k), then S^-1 = L^-T L^-1
    if (tid < D && !failed) {
      const int k = tid;
      for (int i = 0; i < D; ++i) {
        double s = i == k ? 1.0 : 0.0;
        for (int m = k; m < i; ++m) s -= Lc[i][m] * Li[m][k];
        Li[i][k] = i < k ? 0.0 : s / Lc[i][i];
      }
    }
    __syncthreads();
    for (int e = tid; e < D * D; e += kJdThreads) {
      const int k = e / D, l = e - k * D;
      double s = 0.0;
      if (!failed)
        for (int m = max(k, l); m < D; ++m) s += Li[m][k] * Li[m][l];
      Si[k][l] = (float)s;
    }
    __syncthreads();
  }

  // ---- pass 2: depth update, clean-up and covariance of every pixel of frame fr
  float* outr = A.out + fr * HW;
  float* cov = A.dzcov ? A.dzcov + (int64_t)b * HW : nullptr;
  for (int k = tid; k < HW; k += kJdThreads) {
    const int i = k / A.wd, j = k - i * A.wd;
    const int cy = (int)floorf(gy[i]), cx = (int)floorf(gx[j]);
    const Cell c = make_cell(gx[j], gy[i], cx, cy, A.ws);
    const RowTerms r = row_terms(A, b, fr, HW, k, sc_r, c);
    float a = 0.f;
    if (has_src) {
      const float ps = A.prior[fs * HW + k];
      a = ps > 0.f ? ps : 0.f;
    }
    const float dot = c.wt[0] * dso[c.pos[0]] + c.wt[1] * dso[c.pos[1]] + c.wt[2] * dso[c.pos[2]] +
                      c.wt[3] * dso[c.pos[3]];
    const float dz = r.Q * (r.wq + alpha * a * dot);
    outr[k] = jd_clean(r.d + dz);
    if (cov) {
      float quad = 0.f;
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) {
#pragma unroll
        for (int ll = 0; ll < 4; ++ll) quad += c.wt[kk] * c.wt[ll] * Si[c.pos[kk]][c.pos[ll]];
      }
      const float e = alpha * a * r.Q;
      cov[k] = e * e * quad + r.Q;
    }
  }
}

__global__ void __launch_bounds__(kJdThreads)
jdsa_scales_kernel(float* __restrict__ dscales, int D, const int64_t* __restrict__ kx, int M,
                   const float* __restrict__ dso, const int32_t* __restrict__ info) {
  if (*info & (HS2_DEV_BAD_INDEX | HS2_DEV_NOT_PD)) return;
  for (int t = blockIdx.x * kJdThreads + threadIdx.x; t < M * D; t += gridDim.x * kJdThreads) {
    const int b = t / D, k = t - b * D;
    dscales[kx[b] * D + k] += dso[t];
  }
}

}  // namespace
}  // namespace hs2

extern "C" int hs2_jdsa(const float* poses, int64_t num_poses, const float* disps, int64_t num_disps, int ht, int wd,
                        const float* intrinsics, const float* targets, const float* weights, const float* eta,
                        const float* disps_prior, int64_t num_prior, float* dscales, int64_t num_scales, int hs,
                        int ws, const float* grid_y, const float* grid_x, const int64_t* ii, const int64_t* jj,
                        const int64_t* slot, int64_t num_edges, const int64_t* kx, int64_t num_kx, float alpha,
                        float* C, float* w, float* dso, float* disps_out, float* dzcov, int32_t* info,
                        hs2_stream_t stream) {
  using namespace hs2;
  if (num_poses < 0 || num_disps <= 0 || num_disps > 0x7fffffff - 65536 || ht <= 0 || wd <= 0 ||
      ht > kJdMaxAxis || wd > kJdMaxAxis || (int64_t)ht * wd > (1 << 30) || num_prior < 0 || num_scales < 0 ||
      hs < 2 || ws < 2 || hs * ws > kJdMaxD || num_edges < 0 || num_edges > 0x7fffffff) {
    set_error("jdsa: bad sizes (num_disps %lld, ht %d, wd %d, hs %d, ws %d, edges %lld; needs 2 <= hs, ws, "
              "hs*ws <= %d, ht, wd <= %d)", (long long)num_disps, ht, wd, hs, ws, (long long)num_edges, kJdMaxD,
              kJdMaxAxis);
    return HS2_ERR_INVALID;
  }
  if (num_kx <= 0 || num_kx > 65535 || num_kx > num_edges) {
    set_error("jdsa: %lld source frames for %lld edges (the reference indexes kx[0]: at least one edge)",
              (long long)num_kx, (long long)num_edges);
    return HS2_ERR_INVALID;
  }
  if (!grid_y || !grid_x || !kx || !C || !w || !dso || !disps_out || !info) {
    set_error("jdsa: a required pointer is null");
    return HS2_ERR_INVALID;
  }
  int rc = bind_device(disps_out);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  HS2_CUDA(cudaMemsetAsync(info, 0, sizeof(int32_t), s));
  if ((rc = hs2_proj_trans(poses, num_poses, disps, num_disps, ht, wd, intrinsics, targets, weights, ii, jj, slot,
                           num_edges, num_kx, C, w, info, stream)))
    return rc;
  JdArgs A;
  A.disps = disps;
  A.num_disps = num_disps;
  A.ht = ht;
  A.wd = wd;
  A.C = C;
  A.w = w;
  A.eta = eta;
  A.prior = disps_prior;
  A.num_prior = num_prior;
  A.dscales = dscales;
  A.num_scales = num_scales;
  A.hs = hs;
  A.ws = ws;
  A.gy = grid_y;
  A.gx = grid_x;
  A.kx = kx;
  A.M = (int)num_kx;
  A.alpha = alpha;
  A.dso = dso;
  A.out = disps_out;
  A.dzcov = dzcov;
  A.info = info;
  const size_t smem = sizeof(float) * (size_t)(ht + wd);
  HS2_PROF("jdsa_solve", s);
  jdsa_solve_kernel<<<(unsigned)(num_kx + num_disps), kJdThreads, smem, s>>>(A);
  HS2_LAUNCH_CHECK("jdsa_solve_kernel");
  const int D = hs * ws;
  HS2_PROF("jdsa_scales", s);
  jdsa_scales_kernel<<<(unsigned)std::min<int64_t>(64, (num_kx * D + kJdThreads - 1) / kJdThreads), kJdThreads, 0,
                       s>>>(dscales, D, kx, (int)num_kx, dso, info);
  HS2_LAUNCH_CHECK("jdsa_scales_kernel");
  return HS2_OK;
}
