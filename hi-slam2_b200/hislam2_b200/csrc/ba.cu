// Dense bundle adjustment over poses and per-pixel inverse depths
// (reference operator: src/droid.cpp:141-168 -> src/droid_kernels.cu:1820-1937).
//
// One call runs `iterations` damped Gauss-Newton steps entirely on the device:
//
//   keys        unique depth frames kx of cat(arange(t0,t1), ii), edge groups by
//               ii (stable), per-frame row lists of E (reference :1841-1849,
//               :1712-1740, :1413-1439, all host code in the reference)
//   per iteration
//   edge_setup  Gij = Gj Gi^-1 and the 6x6 map L with Ji = L Jj for every edge
//   linearize   per (depth frame, pixel chunk): residuals and Jacobians of all
//               edges leaving that frame; writes the E rows, Q = 1/(C+eta) and w,
//               accumulates each edge's Hjj / vj (reference :364-606, :1901-1906)
//   assemble    Hii = L Hjj L^T, Hij = L Hjj, vi = L vj scattered into the dense
//               FP64 reduced camera matrix (reference update_lhs/update_rhs :1598-1638)
//   schur       per (depth frame, pixel chunk): the Gram of its E rows weighted by
//               Q plus the E.(Q w) column, subtracted from the FP64 system
//               (reference schur_block + EEt6x6 + Ev6x1 :1466-1560, :1689-1779)
//   cholesky    FP64 damped Cholesky + solve, dx = 0 when the factorisation fails
//               (reference SparseBlock::solve :1660-1680)
//   backsub     dz = Q (w - sum_rows E.dx), rows with pose index <= 0 skipped as in
//               the reference (EvT6x1_kernel :1562-1582, :1920), disps += dz
//   pose_retr   poses[t0:t1] <- exp(dx) * poses (FP64 math, reference :1363-1396)
//
// Only the (tiny) key generation is serial; everything else is sized by the
// static problem dimensions, so a whole call is graph-capturable.
//
// The end of the file holds pgba (Sim3 poses, D = 7, one step with relative-pose
// factors), which reuses the keys, the E-row layout and the Cholesky.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <cstdio>
#include <vector>

#include <cuda.h>

#include "ba_common.cuh"
#include "profile.cuh"

namespace hs2 {

constexpr int kLinThreads = 128;
constexpr int kLinPPT = 4;                          // pixels per thread
constexpr int kLinChunk = kLinThreads * kLinPPT;    // pixels per CTA
constexpr int kSchurTP = 32;                        // pixels per smem stage

// ---------------------------------------------------------------- keys ---
// In-place exclusive scan of data[0..n) by one CTA of 1024 threads; returns the total.
// ----------------------------------------------------- frame (fused) ---
// Linearisation and Schur Gram of a depth frame in one kernel: the E rows never leave
// shared memory.  One CTA per (depth frame, pixel split), 288 threads:
//   warps 0-7  per 32-pixel chunk (lane = pixel) warp w linearises edges w, w+8, ... of
//              the frame: residuals, Jacobians, the edge's Hjj / vj (reduced across the
//              warp, kept per edge in registers), partial sums of C, w and the frame's
//              own pose rows, and the E_j rows of Schur edges written raw into the
//              chunk's K-major 128B-swizzled tile.  Targets and weights of the next two
//              chunks are in flight meanwhile (cp.async, three stages; each lane copies
//              and reads only its own values).  After a named barrier of the eight warps
//              they form Q = 1/(C + eta), scale every tile row by sqrt(Q), add the own
//              pose rows and the sqrt(Q) w row, and split the tile into TF32 hi/lo parts;
//   warp 8     allocates TMEM; one lane issues tcgen05.mma kind::tf32 (3xTF32) per chunk
//              for each 128-row M tile against the whole tile, double-buffered through
//              mbarriers; at the end warps 0-7 scatter the Gram from TMEM into the FP64
//              system as ba_schur_tc_kernel does, and each edge's Hjj / vj is added to
//              its FP64 accumulator.
// Frames with more than kFMaxEdges edges or kFMaxRows Schur rows are left to the
// unfused kernels.  Requires Q >= 0 (eta > 0).  Every mbarrier wait is bounded.
constexpr int kFWarps = 8;
constexpr int kFThreads = 32 * (kFWarps + 1);
constexpr int kFK = 32;                                   // pixels per chunk
constexpr int kFMaxEdges = 40;
constexpr int kFSlots = kFMaxEdges / kFWarps;             // edges per warp
constexpr int kFMaxRows = 42;                             // 6 * 42 + 1 <= 256 tile rows
constexpr int kFLd = 3;                                   // cp.async stages
constexpr int kFTile = 256 * 128;                         // 256 rows x 32 fp32
constexpr int kFTiles = 2 * 2 * kFTile;                   // 2 stages x (hi, lo)
constexpr int kFLdBytes = kFLd * kFWarps * kFSlots * 4 * 32 * 4;
constexpr int kFRedBytes = 2 * kFWarps * 8 * 32 * 4;
constexpr int kFTabBytes = kFMaxEdges * kEtab * 4;
constexpr int kFMetaBytes = 1024;
constexpr int kFSmem = 1024 + kFTiles + kFLdBytes + kFRedBytes + kFTabBytes + kFMetaBytes;

__device__ __forceinline__ bool frame_fusable(const BaPtrs& w, int s) {
  return w.gptr[s + 1] - w.gptr[s] <= kFMaxEdges && w.sptr[s + 1] - w.sptr[s] <= kFMaxRows;
}

__device__ int block_exclusive_scan(int* data, int n, int* sh) {
  int carry = 0;
  for (int base = 0; base < n; base += 1024) {
    const int i = base + threadIdx.x;
    int v = i < n ? data[i] : 0;
    // warp inclusive scan
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int s = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int t = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += t;
    }
    if (lane == 31) sh[warp] = s;
    __syncthreads();
    if (warp == 0) {
      int w = sh[lane];
      int ws = w;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, ws, o);
        if (lane >= o) ws += t;
      }
      sh[32 + lane] = ws - w;  // exclusive warp offsets
      if (lane == 31) sh[64] = ws;
    }
    __syncthreads();
    if (i < n) data[i] = carry + sh[32 + warp] + s - v;
    carry += sh[64];
    __syncthreads();
  }
  return carry;
}

__global__ void __launch_bounds__(1024)
ba_keys_kernel(const int64_t* __restrict__ ii, const int64_t* __restrict__ jj, int E, int K, int t0, int t1,
               int64_t eta_rows, BaPtrs w, int32_t* __restrict__ info) {
  __shared__ int sh[72];
  __shared__ int s_bad;
  const int P = t1 - t0;
  if (threadIdx.x == 0) s_bad = 0;
  for (int f = threadIdx.x; f < K; f += 1024) w.slot[f] = 0;
  __syncthreads();
  for (int e = threadIdx.x; e < E; e += 1024) {
    const int64_t a = ii[e], b = jj[e];
    if (a < 0 || b < 0 || a >= K || b >= K || a >= t1 || b >= t1) s_bad = 1;
  }
  __syncthreads();
  if (s_bad) {
    if (threadIdx.x == 0) atomicOr(info, HS2_DEV_BAD_INDEX);
    return;
  }
  for (int e = threadIdx.x; e < E; e += 1024) w.slot[ii[e]] = 1;
  for (int t = t0 + threadIdx.x; t < t1; t += 1024) w.slot[t] = 1;
  __syncthreads();
  // flags -> slot numbers (exclusive scan), kx = inverse
  for (int f = threadIdx.x; f < K; f += 1024) w.flag[f] = w.slot[f];
  __syncthreads();
  const int M = block_exclusive_scan(w.slot, K, sh);
  for (int f = threadIdx.x; f < K; f += 1024) {
    if (w.flag[f]) w.kx[w.slot[f]] = f;
    else w.slot[f] = -1;
  }
  if (threadIdx.x == 0) {
    info[1] = M;
    if (!(eta_rows == M || eta_rows == 1)) {
      atomicOr(info, HS2_DEV_BAD_ETA);
      s_bad = 1;
    }
  }
  __syncthreads();
  if (s_bad) return;
  // edge groups by ii slot: counts, scan, stable fill
  for (int s = threadIdx.x; s <= M; s += 1024) w.gptr[s] = 0;
  __syncthreads();
  for (int e = threadIdx.x; e < E; e += 1024) atomicAdd(&w.gptr[w.slot[ii[e]]], 1);
  __syncthreads();
  block_exclusive_scan(w.gptr, M + 1, sh);
  for (int s = threadIdx.x; s < M; s += 1024) w.cursor[s] = w.gptr[s];
  __syncthreads();
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    for (int base = 0; base < E; base += 32) {
      const int e = base + lane;
      const int key = e < E ? w.slot[ii[e]] : -1 - lane;
      const unsigned mask = __match_any_sync(0xffffffffu, key);
      const int rank = __popc(mask & ((1u << lane) - 1u));
      int pos = 0;
      if (e < E) pos = w.cursor[key] + rank;
      __syncwarp();
      if (e < E) {
        w.gedge[pos] = e;
        if (lane == 31 - __clz(mask)) w.cursor[key] += __popc(mask);
      }
      __syncwarp();
    }
  }
  __syncthreads();
  // row lists per slot: [window row of the frame] + edges of its group
  for (int s = threadIdx.x; s < M; s += 1024) {
    const int f = w.kx[s];
    const int inwin = (f >= t0 && f < t1) ? 1 : 0;
    int ns = inwin;
    for (int g = w.gptr[s]; g < w.gptr[s + 1]; ++g) {
      const int64_t j = jj[w.gedge[g]];
      ns += (j >= t0 && j < t1) ? 1 : 0;
    }
    w.rptr[s] = inwin + (w.gptr[s + 1] - w.gptr[s]);
    w.sptr[s] = ns;
  }
  if (threadIdx.x == 0) { w.rptr[M] = 0; w.sptr[M] = 0; }
  __syncthreads();
  block_exclusive_scan(w.rptr, M + 1, sh);
  block_exclusive_scan(w.sptr, M + 1, sh);
  // E rows are stored depth-frame-major in this list order: a frame's Schur rows
  // first (same order as its srow list), then its rows whose pose is not optimised.
  for (int s = threadIdx.x; s < M; s += 1024) {
    const int f = w.kx[s];
    int r = w.rptr[s], q = w.sptr[s];
    if (f >= t0 && f < t1) {
      w.rrow[r] = f - t0; w.rpose[r] = f - t0; w.wpos[f - t0] = r; ++r;
      w.srow[q] = f - t0; w.spose[q] = f - t0; ++q;
    }
    for (int g = w.gptr[s]; g < w.gptr[s + 1]; ++g) {
      const int e = w.gedge[g];
      const int pj = (int)(jj[e] - t0);
      if (pj >= 0 && pj < P) {
        w.rrow[r] = P + e; w.rpose[r] = pj; w.epos[e] = r; ++r;
        w.srow[q] = P + e; w.spose[q] = pj; ++q;
      }
    }
    for (int g = w.gptr[s]; g < w.gptr[s + 1]; ++g) {
      const int e = w.gedge[g];
      const int pj = (int)(jj[e] - t0);
      if (!(pj >= 0 && pj < P)) { w.rrow[r] = P + e; w.rpose[r] = pj; w.epos[e] = r; ++r; }
    }
  }
}

// kk_exp[n] = slot of ii_exp[n], ii_exp = cat(arange(t0,t1), ii)
__global__ void ba_kk_kernel(const int64_t* __restrict__ ii, int E, int t0, int P, const int* __restrict__ slot,
                             int32_t* __restrict__ kk, const int32_t* __restrict__ info) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= P + E || info[0]) return;
  const int64_t f = n < P ? (int64_t)(t0 + n) : ii[n - P];
  kk[n] = slot[f];
}

// ---------------------------------------------------------- edge setup ---
// Six threads per edge: lane c of the group forms column c of L (the FP64 map Ji = L Jj);
// lane 0 also writes Gij and its rotation matrix.
__device__ __forceinline__ void ba_edge_setup_body(int gid, const float* __restrict__ poses,
                                                   const int64_t* __restrict__ ii, const int64_t* __restrict__ jj,
                                                   int E, float* __restrict__ etab, double* __restrict__ etab64,
                                                   const int32_t* __restrict__ info) {
  const int e = gid / 6, c = gid - (gid / 6) * 6;
  if (e >= E || info[0]) return;
  const int64_t a = ii[e], b = jj[e];
  float tij[3], qij[4];
  relative_pose(poses + 7 * a, poses + 7 * a + 3, poses + 7 * b, poses + 7 * b + 3, tij, qij);
  float* t = etab + (int64_t)e * kEtab;
  if (c == 0) {
    t[0] = tij[0]; t[1] = tij[1]; t[2] = tij[2];
    t[3] = qij[0]; t[4] = qij[1]; t[5] = qij[2]; t[6] = qij[3]; t[7] = 0.f;
    // rotation matrix of qij (row-major) at 44..52
    const float x = qij[0], y = qij[1], z = qij[2], ww = qij[3];
    float* R = t + 44;
    R[0] = 1.f - 2.f * (y * y + z * z); R[1] = 2.f * (x * y - z * ww);       R[2] = 2.f * (x * z + y * ww);
    R[3] = 2.f * (x * y + z * ww);       R[4] = 1.f - 2.f * (x * x + z * z); R[5] = 2.f * (y * z - x * ww);
    R[6] = 2.f * (x * z - y * ww);       R[7] = 2.f * (y * z + x * ww);       R[8] = 1.f - 2.f * (x * x + y * y);
    for (int k = 53; k < kEtab; ++k) t[k] = 0.f;
  }
  const double td[3] = {tij[0], tij[1], tij[2]};
  const double qd[4] = {qij[0], qij[1], qij[2], qij[3]};
  double u[6] = {0, 0, 0, 0, 0, 0};
  u[c] = 1.0;
  double col[6];
  pose_jacobian_i(td, qd, u, col);
  double* L64 = etab64 + (int64_t)e * 36;
  for (int r = 0; r < 6; ++r) {
    L64[r * 6 + c] = col[r];
    t[8 + r * 6 + c] = (float)col[r];
  }
}

__global__ void ba_edge_setup_kernel(const float* __restrict__ poses, const int64_t* __restrict__ ii,
                                     const int64_t* __restrict__ jj, int E, float* __restrict__ etab,
                                     double* __restrict__ etab64, const int32_t* __restrict__ info) {
  ba_edge_setup_body(blockIdx.x * blockDim.x + threadIdx.x, poses, ii, jj, E, etab, etab64, info);
}

// ------------------------------------------------------------ linearize ---
// Sum of v[0..31] over the warp's lanes; lane l returns the total of v[l].  Five
// exchange rounds halve the vector each time (31 shuffles instead of 5 per value).
__device__ __forceinline__ float warp_transpose_sum(float (&v)[32]) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 16, L = 32; o >= 1; o >>= 1, L >>= 1) {
    const bool up = (lane & o) != 0;
#pragma unroll
    for (int i = 0; i < L / 2; ++i) {
      const float send = up ? v[i] : v[i + L / 2];
      const float keep = up ? v[i + L / 2] : v[i];
      v[i] = keep + __shfl_xor_sync(0xffffffffu, send, o);
    }
  }
  return v[0];
}

// One (depth frame s, pixel chunk) of the linearisation on a CTA of NT threads.
template <int NT>
__device__ __forceinline__ void ba_linearize_body(int s, int chunk, const float* __restrict__ disps, int HW, int wd,
                                                  const float* __restrict__ intr, const float* __restrict__ targets,
                                                  const float* __restrict__ weights, const float* __restrict__ eta,
                                                  int64_t eta_rows, const int64_t* __restrict__ jj, int t0, int t1,
                                                  int motion_only, int skip_fusable, BaPtrs w,
                                                  const int32_t* __restrict__ info) {
  constexpr int kChunk = NT * kLinPPT;
  if (info[0]) return;
  const int M = info[1];
  if (s >= M || (skip_fusable && frame_fusable(w, s))) return;
  const int HWs = row_stride(HW);
  const int f = w.kx[s];
  const bool inwin = f >= t0 && f < t1;
  const float fx = intr[0], fy = intr[1], cx = intr[2], cy = intr[3];

  __shared__ float tab[kEtab];
  __shared__ float red[NT / 32][32];

  int pix[kLinPPT];
  float dsp[kLinPPT], xn[kLinPPT], yn[kLinPPT], Cs[kLinPPT], Ws[kLinPPT], Ei[kLinPPT][6];
#pragma unroll
  for (int k = 0; k < kLinPPT; ++k) {
    pix[k] = chunk * kChunk + k * NT + threadIdx.x;
    const int pc = pix[k] < HW ? pix[k] : HW - 1;
    dsp[k] = disps[(int64_t)f * HW + pc];
    const int vi = pc / wd;
    xn[k] = ((float)(pc - vi * wd) - cx) / fx;
    yn[k] = ((float)vi - cy) / fy;
    Cs[k] = 0.f;
    Ws[k] = 0.f;
#pragma unroll
    for (int r = 0; r < 6; ++r) Ei[k][r] = 0.f;
  }

  const int g0 = w.gptr[s], g1 = w.gptr[s + 1];
  for (int g = g0; g < g1; ++g) {
    const int e = w.gedge[g];
    __syncthreads();
    if (threadIdx.x < kEtab) tab[threadIdx.x] = w.etab[(int64_t)e * kEtab + threadIdx.x];
    __syncthreads();
    const bool self = (jj[e] == f);
    const float* trg = targets + (int64_t)e * 2 * HW;
    const float* wgt = weights + (int64_t)e * 2 * HW;
    float* Erow = w.erows + ((int64_t)w.epos[e] * 6) * HWs;
    float tu[kLinPPT], tv[kLinPPT], wgu[kLinPPT], wgv[kLinPPT];
#pragma unroll
    for (int k = 0; k < kLinPPT; ++k) {
      const bool ok = pix[k] < HW;
      tu[k] = ok ? trg[pix[k]] : 0.f;
      tv[k] = ok ? trg[HW + pix[k]] : 0.f;
      wgu[k] = ok ? wgt[pix[k]] : 0.f;
      wgv[k] = ok ? wgt[HW + pix[k]] : 0.f;
    }

    float H[32];
#pragma unroll
    for (int k = 0; k < 32; ++k) H[k] = 0.f;
#pragma unroll
    for (int k = 0; k < kLinPPT; ++k) {
      const int p = pix[k];
      if (p >= HW) continue;
      float Ej[6];
      lin_pixel(tab, fx, fy, cx, cy, xn[k], yn[k], dsp[k], tu[k], tv[k], wgu[k], wgv[k], self,
                H, Cs[k], Ws[k], Ej);
      if (!motion_only) {
#pragma unroll
        for (int r = 0; r < 6; ++r) Erow[(int64_t)r * HWs + p] = Ej[r];
        if (inwin) {
#pragma unroll
          for (int r = 0; r < 6; ++r) {
            float acc = 0.f;
#pragma unroll
            for (int c = 0; c < 6; ++c) acc = fmaf(tab[8 + r * 6 + c], Ej[c], acc);
            Ei[k][r] += acc;
          }
        }
      }
    }
    // block reduction of the 27 Hessian/gradient partial sums of this edge
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    red[warp][lane] = warp_transpose_sum(H);
    __syncthreads();
    if (threadIdx.x < 27) {
      double acc = 0.0;
#pragma unroll
      for (int q2 = 0; q2 < NT / 32; ++q2) acc += (double)red[q2][threadIdx.x];
      atomicAdd(&w.hedge[(int64_t)e * 27 + threadIdx.x], acc);
    }
  }

  if (motion_only) return;
  const float* eta_row = eta + (eta_rows == 1 ? 0 : (int64_t)s * HW);
#pragma unroll
  for (int k = 0; k < kLinPPT; ++k) {
    const int p = pix[k];
    if (p >= HW) continue;
    w.qbuf[(int64_t)s * HW + p] = 1.0f / (Cs[k] + eta_row[p]);
    w.wbuf[(int64_t)s * HW + p] = Ws[k];
    if (inwin) {
      float* Er = w.erows + ((int64_t)w.wpos[f - t0] * 6) * HWs;
#pragma unroll
      for (int r = 0; r < 6; ++r) Er[(int64_t)r * HWs + p] = Ei[k][r];
    }
  }
}

__global__ void __launch_bounds__(kLinThreads, 4)
ba_linearize_kernel(const float* __restrict__ disps, int HW, int wd, const float* __restrict__ intr,
                    const float* __restrict__ targets, const float* __restrict__ weights,
                    const float* __restrict__ eta, int64_t eta_rows, const int64_t* __restrict__ jj,
                    int t0, int t1, int motion_only, int skip_fusable, BaPtrs w,
                    const int32_t* __restrict__ info) {
  ba_linearize_body<kLinThreads>(blockIdx.x, blockIdx.y, disps, HW, wd, intr, targets, weights, eta, eta_rows, jj, t0,
                                 t1, motion_only, skip_fusable, w, info);
}

// ------------------------------------------------------------- assemble ---
// Six threads per edge: lane r of the group adds row r of Hjj / vj (block j), of
// Hii = L Hjj L^T / vi = L vj (block i) and of Hij = L Hjj (lower block triangle).
__device__ __forceinline__ void ba_assemble_body(int gid, const int64_t* __restrict__ ii,
                                                 const int64_t* __restrict__ jj, int E, int t0, int P, BaPtrs w,
                                                 const int32_t* __restrict__ info) {
  const int e = gid / 6, r = gid - (gid / 6) * 6;
  if (e >= E || info[0]) return;
  const int i = (int)(ii[e] - t0), j = (int)(jj[e] - t0);
  if (i < 0 && j < 0) return;
  const double* h = w.hedge + (int64_t)e * 27;
  const double* L = w.etab64 + (int64_t)e * 36;
  double Hjj[6][6], vj[6];
#pragma unroll
  for (int a = 0; a < 6; ++a) {
    vj[a] = h[21 + a];
#pragma unroll
    for (int c = a; c < 6; ++c) Hjj[a][c] = Hjj[c][a] = h[tri6(a, c)];
  }
  const int64_t n = 6 * (int64_t)P;
  double* A = w.A;
  if (j >= 0) {
    atomicAdd(&w.b[j * 6 + r], vj[r]);
#pragma unroll
    for (int c = 0; c < 6; ++c) atomicAdd(&A[(j * 6 + r) * n + j * 6 + c], Hjj[r][c]);
  }
  if (i < 0) return;
  double Lr[6], Hij[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) Lr[k] = L[r * 6 + k];
  double vi = 0.0;
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    double acc = 0.0;
#pragma unroll
    for (int k = 0; k < 6; ++k) acc += Lr[k] * Hjj[k][c];
    Hij[c] = acc;
    vi += Lr[c] * vj[c];
  }
  atomicAdd(&w.b[i * 6 + r], vi);
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    double acc = 0.0;
#pragma unroll
    for (int k = 0; k < 6; ++k) acc += Hij[k] * L[c * 6 + k];
    atomicAdd(&A[(i * 6 + r) * n + i * 6 + c], acc);
  }
  if (j < 0) return;
  // only the lower block triangle of the system is kept (the factorisation reads nothing else)
  if (i > j) {
#pragma unroll
    for (int c = 0; c < 6; ++c) atomicAdd(&A[(i * 6 + r) * n + j * 6 + c], Hij[c]);
  } else if (j > i) {
#pragma unroll
    for (int c = 0; c < 6; ++c) atomicAdd(&A[(j * 6 + c) * n + i * 6 + r], Hij[c]);
  } else {
    // i == j (self edge): Hij + Hij^T on the diagonal block; the transpose row needs the
    // other lanes' Hij, formed here from L and Hjj directly
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      double tcr = 0.0;
#pragma unroll
      for (int k = 0; k < 6; ++k) tcr += L[c * 6 + k] * Hjj[k][r];
      atomicAdd(&A[(i * 6 + r) * n + i * 6 + c], Hij[c] + tcr);
    }
  }
}

__global__ void ba_assemble_kernel(const int64_t* __restrict__ ii, const int64_t* __restrict__ jj, int E, int t0,
                                   int P, BaPtrs w, const int32_t* __restrict__ info) {
  ba_assemble_body(blockIdx.x * blockDim.x + threadIdx.x, ii, jj, E, t0, P, w, info);
}

// ---------------------------------------------------------------- schur ---
// Per (depth frame k, pixel chunk): S_ab = sum_p Q E_a E_b^T for every pair of the
// frame's Schur rows a <= b (6x6 blocks) and v_a = sum_p Q w E_a.  Rows are
// processed in tiles of kSchurTB blocks; a CTA thread owns up to two items (a
// block pair or a w pair) and keeps their 36 sums in registers while the rows'
// values for 32 pixels at a time sit in shared memory.  Results go to the lower
// triangle of the FP64 reduced camera system (all that the factorisation reads):
// S_ab lands on block (pose_a, pose_b) when pose_a > pose_b and transposed on
// (pose_b, pose_a) otherwise.
constexpr int kSchurTB = 22;                 // row blocks per tile
constexpr int kSchurTR = 6 * kSchurTB;       // rows per tile
constexpr int kSchurItems = 2;               // items per thread

__device__ __forceinline__ void schur_scatter_block(double* A, int64_t n, int pa, int pb, bool same_row,
                                                    const float (&acc)[36]) {
  if (pa > pb) {
#pragma unroll
    for (int x = 0; x < 6; ++x)
#pragma unroll
      for (int y = 0; y < 6; ++y) atomicAdd(&A[(pa * 6 + x) * n + pb * 6 + y], -(double)acc[x * 6 + y]);
  } else if (pa < pb) {
#pragma unroll
    for (int x = 0; x < 6; ++x)
#pragma unroll
      for (int y = 0; y < 6; ++y) atomicAdd(&A[(pb * 6 + y) * n + pa * 6 + x], -(double)acc[x * 6 + y]);
  } else {
    // same pose: S_ab (+ S_ab^T for two different rows) on the diagonal block
#pragma unroll
    for (int x = 0; x < 6; ++x)
#pragma unroll
      for (int y = 0; y < 6; ++y) {
        double v = -(double)acc[x * 6 + y];
        if (!same_row) v -= (double)acc[y * 6 + x];
        atomicAdd(&A[(pa * 6 + x) * n + pa * 6 + y], v);
      }
  }
}

// One (depth frame s, pixel split) of the SIMT Schur Gram on a CTA of 256 threads.
__device__ __forceinline__ void ba_schur_body(int s, int split, int HW, int chunk, BaPtrs w, int P, int min_blocks,
                                              int skip_fusable, const int32_t* __restrict__ info) {
  if (info[0]) return;
  if (s >= info[1] || (skip_fusable && frame_fusable(w, s))) return;
  const int r0 = w.sptr[s];
  const int nr = w.sptr[s + 1] - r0;
  if (nr == 0 || nr < min_blocks) return;
  const int c0 = split * chunk;
  const int c1 = min(HW, c0 + chunk);
  if (c0 >= c1) return;
  const int* spose = w.spose + r0;
  const int rbase = w.rptr[s];          // storage position of the frame's first Schur row
  const int HWs = row_stride(HW);
  const int64_t n = 6 * (int64_t)P;
  const float* Q = w.qbuf + (int64_t)s * HW;
  const float* W = w.wbuf + (int64_t)s * HW;

  __shared__ float Fa[kSchurTP][kSchurTR + 2];   // Q-scaled rows of tile mt
  __shared__ float Fb[kSchurTP][kSchurTR + 2];   // rows of tile nt
  __shared__ float Ws[kSchurTP];

  const int ntile = (nr + kSchurTB - 1) / kSchurTB;
  for (int mt = 0; mt < ntile; ++mt) {
    for (int nt = mt; nt < ntile; ++nt) {
      const int na = min(kSchurTB, nr - mt * kSchurTB);
      const int nb = min(kSchurTB, nr - nt * kSchurTB);
      const bool diag = mt == nt;
      const int npairs = diag ? na * (na + 1) / 2 : na * nb;
      const int nitems = npairs + (diag ? na : 0);
      int ia[kSchurItems], ib[kSchurItems];   // ib == -1: w pair
      bool live[kSchurItems];
#pragma unroll
      for (int q = 0; q < kSchurItems; ++q) {
        const int it = threadIdx.x + q * 256;
        live[q] = it < nitems;
        ia[q] = 0;
        ib[q] = -1;
        if (it < npairs) {
          if (diag) {
            // it -> (a, b) with a <= b, row-major over the upper triangle
            int a = 0, rem = it;
            while (rem >= na - a) { rem -= na - a; ++a; }
            ia[q] = a;
            ib[q] = a + rem;
          } else {
            ia[q] = it / nb;
            ib[q] = it - (it / nb) * nb;
          }
        } else if (it < nitems) {
          ia[q] = it - npairs;
        }
      }
      float acc[kSchurItems][36];
#pragma unroll
      for (int q = 0; q < kSchurItems; ++q)
#pragma unroll
        for (int k = 0; k < 36; ++k) acc[q][k] = 0.f;

      for (int p0 = c0; p0 < c1; p0 += kSchurTP) {
        __syncthreads();
        for (int idx = threadIdx.x; idx < kSchurTR * kSchurTP; idx += 256) {
          const int row = idx / kSchurTP;
          const int pp = idx - row * kSchurTP;
          const int p = p0 + pp;
          const int blk = row / 6, d = row - (row / 6) * 6;
          float va = 0.f, vb = 0.f;
          if (p < c1) {
            if (blk < na) va = w.erows[((int64_t)(rbase + mt * kSchurTB + blk) * 6 + d) * HWs + p] * Q[p];
            if (blk < nb) vb = w.erows[((int64_t)(rbase + nt * kSchurTB + blk) * 6 + d) * HWs + p];
          }
          Fa[pp][row] = va;
          Fb[pp][row] = vb;
        }
        if (threadIdx.x < kSchurTP) {
          const int p = p0 + threadIdx.x;
          Ws[threadIdx.x] = p < c1 ? W[p] : 0.f;
        }
        __syncthreads();
#pragma unroll 2
        for (int pp = 0; pp < kSchurTP; ++pp) {
#pragma unroll
          for (int q = 0; q < kSchurItems; ++q) {
            if (!live[q]) continue;
            float av[6];
#pragma unroll
            for (int x = 0; x < 6; ++x) av[x] = Fa[pp][ia[q] * 6 + x];
            if (ib[q] >= 0) {
              float bv[6];
#pragma unroll
              for (int y = 0; y < 6; ++y) bv[y] = Fb[pp][ib[q] * 6 + y];
#pragma unroll
              for (int x = 0; x < 6; ++x)
#pragma unroll
                for (int y = 0; y < 6; ++y) acc[q][x * 6 + y] += av[x] * bv[y];
            } else {
              const float wv = Ws[pp];
#pragma unroll
              for (int x = 0; x < 6; ++x) acc[q][x] += av[x] * wv;
            }
          }
        }
      }
#pragma unroll
      for (int q = 0; q < kSchurItems; ++q) {
        if (!live[q]) continue;
        const int ra = mt * kSchurTB + ia[q];
        const int pa = spose[ra];
        if (ib[q] >= 0) {
          const int rb = nt * kSchurTB + ib[q];
          schur_scatter_block(w.A, n, pa, spose[rb], ra == rb, acc[q]);
        } else {
#pragma unroll
          for (int x = 0; x < 6; ++x) atomicAdd(&w.b[pa * 6 + x], -(double)acc[q][x]);
        }
      }
    }
  }
}

__global__ void __launch_bounds__(256)
ba_schur_kernel(int HW, int chunk, BaPtrs w, int P, int min_blocks, int skip_fusable,
                const int32_t* __restrict__ info) {
  ba_schur_body(blockIdx.x, blockIdx.y, HW, chunk, w, P, min_blocks, skip_fusable, info);
}

// Mirrors the lower triangle of the reduced system into the upper one (diagnostics only).
__global__ void ba_symmetrize_kernel(int n, double* __restrict__ A) {
  const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (idx >= (int64_t)n * n) return;
  const int i = (int)(idx / n), j = (int)(idx - (idx / n) * n);
  if (j > i) A[idx] = A[(int64_t)j * n + i];
}

// ------------------------------------------------------- schur (tcgen05) ---
// Tensor-core form of the Schur Gram.  With G = sqrt(Q) o F (the frame's Schur rows
// scaled per pixel) the frame's block of the Gram is S = G G^T and its rhs column is
// v = G (sqrt(Q) w): one symmetric GEMM per depth frame with K = pixels, B = [G; sqrt(Q) w]
// and A = the one or two 128-row windows of the same shared-memory tile (both held in
// TMEM, so the tile is loaded and split once).  One CTA per (frame, pixel split):
//   warp 9     TMA: per 32-pixel chunk, up to four 64x32 fp32 boxes of the frame's E
//              planes (stored contiguously, depth-frame-major) land 128B-swizzled in
//              the stage's hi tile (cp.async.bulk.tensor, mbarrier complete_tx);
//   warps 0-7  scale by sqrt(Q), add the w row, zero the padding and split each value
//              into TF32 hi/lo parts in place (8 rows in flight per thread);
//   warp 8     allocates 512 TMEM columns; one lane issues tcgen05.mma kind::tf32
//              M=128, N=Npad, K=8: A_hi.B_hi + A_hi.B_lo + A_lo.B_hi (3xTF32) and
//              tcgen05.commit releases the stage / finally signals the epilogue;
//   warps 0-7  read the accumulator (warp w: TMEM lanes of quarter w%4, column half w/4)
//              and scatter the a <= b block pairs and the v column into the lower
//              triangle of the FP64 system.
// Six stages of 32 KB for frames of at most 128 tile rows, else three of 64 KB; every
// mbarrier wait is bounded (HS2_DEV_TIMEOUT).  Frames with
// more than kTcMaxBlocks Schur rows are left to the SIMT kernel.  Requires Q >= 0 (eta > 0).
constexpr int kTcThreads = 320;
constexpr int kTcSplitWarps = 8;
constexpr int kTcK = 32;                       // pixels per stage (128 B per plane row)
constexpr int kTcMaxStages = 6;                // stages of frames of <= 128 tile rows
constexpr int kTcSkip = 112;                   // Gram columns M tile 1 leaves out (<= 126, 16-aligned)
// Schur rows of D values per frame on the tensor cores: N = D * rows + 1 <= 256
__host__ __device__ constexpr int tc_max_blocks(int D) { return 255 / D; }
constexpr int kTcMaxBlocks = tc_max_blocks(6);  // 42 for the SE3 rows of ba
constexpr int kTcRows = 256;                   // plane rows per tile
constexpr int kTcBox = 64;                     // plane rows per TMA box
constexpr int kTcTile = kTcRows * kTcK * 4;    // 32 KB
constexpr int kTcStageBytes = 2 * kTcTile;     // hi + lo
constexpr int kTcArea = 3 * kTcStageBytes;      // 192 KB: 3 stages of 256 rows or 6 of 128
constexpr int kTcSmem = kTcArea + 1024 /*align*/ + 2048 /*barriers*/;
constexpr unsigned kTcSpin = 1u << 26;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint32_t bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(bar),
               "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_test(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
  return ok != 0;
}
// Bounded wait; gives up (and raises *abort) after kTcSpin polls or when another
// thread of the CTA already gave up.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort) {
  for (unsigned i = 0; i < kTcSpin; ++i) {
    if (mbar_test(bar, parity)) return true;
    if (*abort) return false;
  }
  *abort = 1;
  return false;
}
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
      ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar) : "memory");
}
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t saddr) {
  // K-major, 128B swizzle: LBO = 16 B (unused), SBO = 1024 B (8 rows x 128 B), version 1
  uint64_t d = 0;
  d |= (uint64_t)((saddr & 0x3FFFF) >> 4);
  d |= (uint64_t)1 << 16;
  d |= (uint64_t)(1024 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
  return d;
}
__device__ __forceinline__ uint32_t umma_idesc_tf32(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
__device__ __forceinline__ void umma_tf32(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
      ::"r"(tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
}
__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ float tf32_hi(float x) { return __uint_as_float(__float_as_uint(x) & 0xFFFFE000u); }
// byte offset of (row r, pixel k) in a K-major 128B-swizzled tile (1024-byte aligned)
__device__ __forceinline__ uint32_t sw128_off(int r, int k) {
  return (uint32_t)(r * 128 + ((((k >> 2) ^ (r & 7)) & 7) << 4) + ((k & 3) << 2));
}

template <int D>
__global__ void __launch_bounds__(kTcThreads, 1)
ba_schur_tc_kernel(const __grid_constant__ CUtensorMap emap, int HW, int chunk, BaPtrs w, int64_t lda,
                   int32_t* __restrict__ info, int split3) {
  if (info[0]) return;
  const int s = blockIdx.x;
  if (s >= info[1]) return;
  const int nr = w.sptr[s + 1] - w.sptr[s];
  if (nr == 0 || nr > tc_max_blocks(D)) return;
  const int mtiles = (D * nr + 127) / 128;          // 128-row M tiles, both in this CTA
  const int c0 = blockIdx.z * chunk;
  const int c1 = min(HW, c0 + chunk);
  if (c0 >= c1) return;
  const int nrowB = D * nr + 1;                   // + the sqrt(Q) w row
  const int Npad = (nrowB + 15) & ~15;
  const int nbox = (D * nr + kTcBox - 1) / kTcBox;
  const int nchunks = (c1 - c0 + kTcK - 1) / kTcK;
  const int prow0 = w.rptr[s] * D;                 // first plane row of the frame's Schur rows

  extern __shared__ uint8_t tc_raw[];
  const uint32_t raw = smem_u32(tc_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  uint8_t* gbase = tc_raw + (base - raw);
  uint8_t* meta = gbase + kTcArea;
  uint64_t* bars = reinterpret_cast<uint64_t*>(meta);  // tma[3], full[3], empty[3], done
  volatile int* abort_flag = reinterpret_cast<volatile int*>(meta + 256);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(meta + 264);
  const uint32_t bar_tma = smem_u32(bars), bar_full = smem_u32(bars + kTcMaxStages);
  const uint32_t bar_empty = smem_u32(bars + 2 * kTcMaxStages), bar_done = smem_u32(bars + 3 * kTcMaxStages);
  // tile rows: 128 when the frame's rows fit (twice the stages in flight), else 256
  const int trows = Npad <= 128 ? 128 : kTcRows;
  const uint32_t tile_bytes = (uint32_t)trows * 128u, stage_bytes = 2u * tile_bytes;
  const int nst = kTcArea / (int)stage_bytes;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int* spose = w.spose + w.sptr[s];
  if (tid == 0) {
    for (int q = 0; q < nst; ++q) {
      mbar_init(bar_tma + 8 * q, 1);
      mbar_init(bar_full + 8 * q, kTcSplitWarps);
      mbar_init(bar_empty + 8 * q, 1);
    }
    mbar_init(bar_done, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == kTcSplitWarps) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(512) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const float* Q = w.qbuf + (int64_t)s * HW;
  const float* Wv = w.wbuf + (int64_t)s * HW;

  if (warp == kTcSplitWarps + 1) {
    // ------------------------------------------------------------- TMA producer
    if (lane == 0) {
      const uint32_t bytes = (uint32_t)nbox * kTcBox * kTcK * 4;
      for (int c = 0; c < nchunks; ++c) {
        const int st = c % nst;
        const int use = c / nst;
        if (use > 0 && !mbar_wait(bar_empty + 8 * st, (use - 1) & 1, abort_flag)) break;
        mbar_arrive_tx(bar_tma + 8 * st, bytes);
        const uint32_t dst = base + st * stage_bytes;
        for (int i = 0; i < nbox; ++i)
          tma_load_2d(dst + i * kTcBox * 128, &emap, c0 + c * kTcK, prow0 + i * kTcBox, bar_tma + 8 * st);
      }
    }
  } else if (warp < kTcSplitWarps) {
    // ------------------------------------------------------------- split
    int pn = c0 + lane;
    float qn = pn < c1 ? Q[pn] : 0.f, wn = pn < c1 ? Wv[pn] : 0.f;
    for (int c = 0; c < nchunks; ++c) {
      const int st = c % nst;
      const float sq = sqrtf(fmaxf(qn, 0.f));
      const float wq = wn * sq;
      // prefetch Q, w of the next chunk
      pn = c0 + (c + 1) * kTcK + lane;
      qn = pn < c1 ? Q[pn] : 0.f;
      wn = pn < c1 ? Wv[pn] : 0.f;
      if (!mbar_wait(bar_tma + 8 * st, (c / nst) & 1, abort_flag)) break;
      uint8_t* hi = gbase + st * stage_bytes;
      uint8_t* lo = hi + tile_bytes;
      for (int rb = warp; rb < Npad; rb += 8 * kTcSplitWarps) {
        float g[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const int r = rb + u * kTcSplitWarps;
          float v = 0.f;
          if (r < D * nr) v = *reinterpret_cast<const float*>(hi + sw128_off(r, lane)) * sq;
          else if (r == D * nr) v = wq;
          g[u] = v;
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const int r = rb + u * kTcSplitWarps;
          if (r < Npad) {
            const uint32_t o = sw128_off(r, lane);
            if (split3) {
              const float gh = tf32_hi(g[u]);
              *reinterpret_cast<float*>(hi + o) = gh;
              *reinterpret_cast<float*>(lo + o) = g[u] - gh;
            } else {
              *reinterpret_cast<float*>(hi + o) = g[u];   // one TF32 product: the MMA reads the top bits
            }
          }
        }
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(bar_full + 8 * st);
    }
  } else if (lane == 0) {
    // ------------------------------------------------------------- MMA issuer
    // M tile 1 (rows >= 128) only needs the columns of blocks b >= a >= 128 / D, i.e. from 126 on:
    // its B operand starts at row kTcSkip (a multiple of 8 rows, N stays a multiple of 16)
    const uint32_t idesc0 = umma_idesc_tf32(128, Npad), idesc1 = umma_idesc_tf32(128, Npad - kTcSkip);
    for (int c = 0; c < nchunks; ++c) {
      const int st = c % nst;
      if (!mbar_wait(bar_full + 8 * st, (c / nst) & 1, abort_flag)) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t b_hi = base + st * stage_bytes;
      const uint32_t b_lo = b_hi + tile_bytes;
      for (int mt = 0; mt < mtiles; ++mt) {
        const uint32_t a_hi = b_hi + mt * 128 * 128;
        const uint32_t a_lo = b_lo + mt * 128 * 128;
        const uint32_t boff = mt ? kTcSkip * 128u : 0u;
        const uint32_t idesc = mt ? idesc1 : idesc0;
        const uint32_t d = tmem + (uint32_t)(mt * Npad);
#pragma unroll
        for (int k = 0; k < kTcK / 8; ++k) {
          const uint32_t kb = k * 32;
          umma_tf32(d, umma_desc_sw128(a_hi + kb), umma_desc_sw128(b_hi + boff + kb), idesc, (c | k) ? 1u : 0u);
          if (split3) {
            umma_tf32(d, umma_desc_sw128(a_hi + kb), umma_desc_sw128(b_lo + boff + kb), idesc, 1u);
            umma_tf32(d, umma_desc_sw128(a_lo + kb), umma_desc_sw128(b_hi + boff + kb), idesc, 1u);
          }
        }
      }
      umma_commit(bar_empty + 8 * st);
    }
    umma_commit(bar_done);
  }

  // ------------------------------------------------------------- epilogue
  if (warp < kTcSplitWarps) {
    const bool ok = mbar_wait(bar_done, 0, abort_flag);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int quarter = warp & 3;                    // TMEM lane quarter of this warp
    const int64_t n = lda;
    for (int mt = 0; mt < mtiles; ++mt) {
      const int R = mt * 128 + quarter * 32 + lane;  // plane row of this accumulator row
      const bool mrow = ok && R < D * nr;
      const int a = R / D, x = R % D;
      const int pa = mrow ? spose[a] : 0;
      const int cbase = mt ? kTcSkip : 0;             // first Gram column held by this M tile
      for (int col0 = (warp >> 2) * 16; cbase + col0 < Npad; col0 += 32) {
        uint32_t v[16];
        const uint32_t taddr = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(mt * Npad + col0);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
              "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (!mrow) continue;
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int col = cbase + col0 + j;
          const double val = -(double)__uint_as_float(v[j]);
          if (col < D * nr) {
            const int b = col / D, y = col % D;
            if (b < a) continue;
            const int pb = spose[b];
            if (pa > pb) atomicAdd(&w.A[(pa * D + x) * n + pb * D + y], val);
            else if (pa < pb) atomicAdd(&w.A[(pb * D + y) * n + pa * D + x], val);
            else {
              atomicAdd(&w.A[(pa * D + x) * n + pa * D + y], val);
              if (a != b) atomicAdd(&w.A[(pa * D + y) * n + pa * D + x], val);
            }
          } else if (col == D * nr) {
            atomicAdd(&w.b[pa * D + x], val);
          }
        }
      }
    }
  }
  if (*abort_flag && tid == 0) atomicOr(info, HS2_DEV_TIMEOUT);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == kTcSplitWarps) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512) : "memory");
  }
}

__device__ __forceinline__ void cp_async4(uint32_t dst, const float* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(dst), "l"(src) : "memory");
}

__global__ void __launch_bounds__(kFThreads, 1)
ba_frame_kernel(const float* __restrict__ disps, int HW, int wd, const float* __restrict__ intr,
                const float* __restrict__ targets, const float* __restrict__ weights,
                const float* __restrict__ eta, int64_t eta_rows, const int64_t* __restrict__ jj, int t0, int t1,
                int chunk, BaPtrs w, int32_t* __restrict__ info) {
  if (info[0]) return;
  const int s = blockIdx.x;
  if (s >= info[1] || !frame_fusable(w, s)) return;
  const int c0 = blockIdx.y * chunk;
  const int c1 = min(HW, c0 + chunk);
  if (c0 >= c1) return;
  const int P = t1 - t0;
  const int f = w.kx[s];
  const bool inwin = f >= t0 && f < t1;
  const int g0 = w.gptr[s], ne = w.gptr[s + 1] - g0;
  const int nr = w.sptr[s + 1] - w.sptr[s];
  const int rbase = w.rptr[s];
  const int own = inwin ? w.wpos[f - t0] - rbase : -1;     // Schur row of the frame's own pose
  const bool gram = nr > 0;
  const int nrow = 6 * nr;
  const int Npad = (nrow + 1 + 15) & ~15;
  const int mtiles = (nrow + 127) / 128;
  const int nchunks = (c1 - c0 + kFK - 1) / kFK;
  const float fx = intr[0], fy = intr[1], cx = intr[2], cy = intr[3];

  extern __shared__ uint8_t f_raw[];
  const uint32_t raw = smem_u32(f_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  uint8_t* gb = f_raw + (base - raw);
  uint8_t* tiles = gb;                                                  // [2][hi, lo]
  float* ldbuf = reinterpret_cast<float*>(gb + kFTiles);               // [kFLd][8][kFSlots][4][32]
  float* red = reinterpret_cast<float*>(gb + kFTiles + kFLdBytes);     // [2][8][8][32]
  float* tab = reinterpret_cast<float*>(gb + kFTiles + kFLdBytes + kFRedBytes);   // [kFMaxEdges][48]
  uint8_t* meta = gb + kFTiles + kFLdBytes + kFRedBytes + kFTabBytes;
  uint64_t* bars = reinterpret_cast<uint64_t*>(meta);                  // full[2], empty[2], done
  int* erow = reinterpret_cast<int*>(meta + 64);                        // [kFMaxEdges] Schur row or -1
  int* eself = erow + kFMaxEdges;                                       // [kFMaxEdges]
  volatile int* abort_flag = reinterpret_cast<volatile int*>(meta + 512);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(meta + 520);
  const uint32_t bar_full = smem_u32(bars), bar_empty = smem_u32(bars + 2), bar_done = smem_u32(bars + 4);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int i = tid; i < ne * kEtab; i += kFThreads) tab[i] = w.etab[(int64_t)w.gedge[g0 + i / kEtab] * kEtab + i % kEtab];
  if (tid < ne) {
    const int e = w.gedge[g0 + tid];
    const int q = w.epos[e] - rbase;
    erow[tid] = q < nr ? q : -1;
    eself[tid] = jj[e] == f;
  }
  if (tid == 0) {
    for (int q = 0; q < 2; ++q) {
      mbar_init(bar_full + 8 * q, kFWarps);
      mbar_init(bar_empty + 8 * q, 1);
    }
    mbar_init(bar_done, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == kFWarps && gram) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(512) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = gram ? *tmem_slot : 0u;

  if (warp < kFWarps) {
    // ------------------------------------------------------------- linearise
    const float* Qeta = eta + (eta_rows == 1 ? 0 : (int64_t)s * HW);
    float hacc[kFSlots];
#pragma unroll
    for (int k = 0; k < kFSlots; ++k) hacc[k] = 0.f;
    float* myld = ldbuf + (warp * kFSlots * 4) * 32 + lane;           // + stage * 8*kFSlots*128, + (k*4+a)*32
    auto issue = [&](int c) {
      if (c < nchunks) {
        const int st = c % kFLd;
        const int p = c0 + c * kFK + lane;
        if (p < c1) {
#pragma unroll
          for (int k = 0; k < kFSlots; ++k) {
            const int el = warp + kFWarps * k;
            if (el < ne) {
              const int64_t e = w.gedge[g0 + el];
              const uint32_t dst = smem_u32(myld + st * (kFWarps * kFSlots * 128) + k * 128);
              cp_async4(dst, targets + e * 2 * HW + p);
              cp_async4(dst + 128, targets + e * 2 * HW + HW + p);
              cp_async4(dst + 256, weights + e * 2 * HW + p);
              cp_async4(dst + 384, weights + e * 2 * HW + HW + p);
            }
          }
        }
      }
      asm volatile("cp.async.commit_group;" ::: "memory");
    };
    issue(0);
    issue(1);
    bool ok = true;
    for (int c = 0; c < nchunks; ++c) {
      issue(c + 2);
      asm volatile("cp.async.wait_group 2;" ::: "memory");
      const int st = c % kFLd;
      const int p = c0 + c * kFK + lane;
      const bool valid = p < c1;
      const int pc = valid ? p : c1 - 1;
      const int vi = pc / wd;
      const float xn = ((float)(pc - vi * wd) - cx) / fx, yn = ((float)vi - cy) / fy;
      const float h = disps[(int64_t)f * HW + pc];
      const int tb = c & 1;
      uint8_t* thi = tiles + tb * 2 * kFTile;
      uint8_t* tlo = thi + kFTile;
      if (gram && c >= 2) ok = ok && mbar_wait(bar_empty + 8 * tb, ((c - 2) >> 1) & 1, abort_flag);
      float cs = 0.f, ws = 0.f, ei[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
      for (int k = 0; k < kFSlots; ++k) {
        const int el = warp + kFWarps * k;
        if (el >= ne) break;
        const float* tl = tab + el * kEtab;
        const float* ld = myld + st * (kFWarps * kFSlots * 128) + k * 128;
        const float tu = valid ? ld[0] : 0.f, tv = valid ? ld[32] : 0.f;
        const float wgu = valid ? ld[64] : 0.f, wgv = valid ? ld[96] : 0.f;
        float H[32];
#pragma unroll
        for (int i = 0; i < 32; ++i) H[i] = 0.f;
        float Ej[6];
        lin_pixel(tl, fx, fy, cx, cy, xn, yn, h, tu, tv, wgu, wgv, eself[el] != 0, H, cs, ws, Ej);
        hacc[k] += warp_transpose_sum(H);
        const int q = erow[el];
        if (gram && q >= 0) {
#pragma unroll
          for (int r = 0; r < 6; ++r) *reinterpret_cast<float*>(thi + sw128_off(6 * q + r, lane)) = Ej[r];
        }
        if (inwin) {
#pragma unroll
          for (int r = 0; r < 6; ++r) {
            float acc = 0.f;
#pragma unroll
            for (int cc = 0; cc < 6; ++cc) acc += tl[8 + r * 6 + cc] * Ej[cc];
            ei[r] += acc;
          }
        }
      }
      float* rd = red + tb * (kFWarps * 8 * 32);
      rd[(warp * 8 + 0) * 32 + lane] = cs;
      rd[(warp * 8 + 1) * 32 + lane] = ws;
#pragma unroll
      for (int r = 0; r < 6; ++r) rd[(warp * 8 + 2 + r) * 32 + lane] = ei[r];
      asm volatile("bar.sync 1, %0;" ::"r"(kFWarps * 32) : "memory");
      float ct = 0.f, wt = 0.f;
#pragma unroll
      for (int q = 0; q < kFWarps; ++q) {
        ct += rd[(q * 8 + 0) * 32 + lane];
        wt += rd[(q * 8 + 1) * 32 + lane];
      }
      const float Qp = valid ? 1.0f / (ct + Qeta[pc]) : 0.f;
      if (warp == 0 && valid) {
        w.qbuf[(int64_t)s * HW + p] = Qp;
        w.wbuf[(int64_t)s * HW + p] = wt;
      }
      if (gram) {
        const float sq = sqrtf(fmaxf(Qp, 0.f));
        for (int r = warp; r < Npad; r += kFWarps) {
          float g = 0.f;
          if (r < nrow) {
            const int a = r / 6;
            float val;
            if (a == own) {
              val = 0.f;
#pragma unroll
              for (int q = 0; q < kFWarps; ++q) val += rd[(q * 8 + 2 + (r - 6 * a)) * 32 + lane];
            } else {
              val = *reinterpret_cast<const float*>(thi + sw128_off(r, lane));
            }
            g = val * sq;
          } else if (r == nrow) {
            g = wt * sq;
          }
          const uint32_t o = sw128_off(r, lane);
          const float gh = tf32_hi(g);
          *reinterpret_cast<float*>(thi + o) = gh;
          *reinterpret_cast<float*>(tlo + o) = g - gh;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncwarp();
        if (lane == 0) mbar_arrive(bar_full + 8 * tb);
      }
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    // each edge's Hjj / vj
#pragma unroll
    for (int k = 0; k < kFSlots; ++k) {
      const int el = warp + kFWarps * k;
      if (el < ne && lane < 27) atomicAdd(&w.hedge[(int64_t)w.gedge[g0 + el] * 27 + lane], (double)hacc[k]);
    }
    (void)ok;
  } else if (gram && lane == 0) {
    // ------------------------------------------------------------- MMA issuer
    const uint32_t idesc = umma_idesc_tf32(128, Npad);
    for (int c = 0; c < nchunks; ++c) {
      const int tb = c & 1;
      if (!mbar_wait(bar_full + 8 * tb, (c >> 1) & 1, abort_flag)) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t b_hi = base + tb * 2 * kFTile;
      const uint32_t b_lo = b_hi + kFTile;
      for (int mt = 0; mt < mtiles; ++mt) {
        const uint32_t a_hi = b_hi + mt * 128 * 128, a_lo = b_lo + mt * 128 * 128;
        const uint32_t d = tmem + (uint32_t)(mt * Npad);
#pragma unroll
        for (int k = 0; k < kFK / 8; ++k) {
          const uint32_t kb = k * 32;
          umma_tf32(d, umma_desc_sw128(a_hi + kb), umma_desc_sw128(b_hi + kb), idesc, (c | k) ? 1u : 0u);
          umma_tf32(d, umma_desc_sw128(a_hi + kb), umma_desc_sw128(b_lo + kb), idesc, 1u);
          umma_tf32(d, umma_desc_sw128(a_lo + kb), umma_desc_sw128(b_hi + kb), idesc, 1u);
        }
      }
      umma_commit(bar_empty + 8 * tb);
    }
    umma_commit(bar_done);
  }

  // ------------------------------------------------------------- Gram scatter
  if (gram && warp < kFWarps) {
    const bool ok = mbar_wait(bar_done, 0, abort_flag);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int64_t n = 6 * (int64_t)P;
    const int* spose = w.spose + w.sptr[s];
    const int quarter = warp & 3;
    for (int mt = 0; mt < mtiles; ++mt) {
      const int R = mt * 128 + quarter * 32 + lane;
      const bool mrow = ok && R < nrow;
      const int a = R / 6, x = R % 6;
      const int pa = mrow ? spose[a] : 0;
      for (int col0 = (warp >> 2) * 16; col0 < Npad; col0 += 32) {
        uint32_t v[16];
        const uint32_t taddr = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(mt * Npad + col0);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
              "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (!mrow) continue;
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int col = col0 + j;
          const double val = -(double)__uint_as_float(v[j]);
          if (col < nrow) {
            const int b = col / 6, y = col % 6;
            if (b < a) continue;
            const int pb = spose[b];
            if (pa > pb) atomicAdd(&w.A[(pa * 6 + x) * n + pb * 6 + y], val);
            else if (pa < pb) atomicAdd(&w.A[(pb * 6 + y) * n + pa * 6 + x], val);
            else {
              atomicAdd(&w.A[(pa * 6 + x) * n + pa * 6 + y], val);
              if (a != b) atomicAdd(&w.A[(pa * 6 + y) * n + pa * 6 + x], val);
            }
          } else if (col == nrow) {
            atomicAdd(&w.b[pa * 6 + x], val);
          }
        }
      }
    }
  }
  if (*abort_flag && tid == 0) atomicOr(info, HS2_DEV_TIMEOUT);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == kFWarps && gram) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512) : "memory");
  }
}

// Back-substitution with the E rows recomputed from the weights (the fused path keeps
// none): per pixel of depth frame f, dz = Q (w - sum_e E_j(e) . u_e) with
// u_e = dx_j + L_e^T dx_f, each term present only when its pose index lies in (0, P)
// as in the reference's EvT6x1 (the frame's own row E_f = sum_e L_e E_j(e)).
__global__ void __launch_bounds__(kLinThreads)
ba_backsub_frame_kernel(float* __restrict__ disps, int HW, int wd, const float* __restrict__ intr,
                        const float* __restrict__ weights, const int64_t* __restrict__ jj, int t0, int t1,
                        BaPtrs w, const float* __restrict__ dx, float* __restrict__ dz, int64_t dz_rows,
                        const int32_t* __restrict__ info) {
  if (info[0]) return;
  const int s = blockIdx.x;
  if (s >= info[1] || s >= dz_rows) return;
  const int P = t1 - t0;
  const int f = w.kx[s];
  const int fi = f - t0;
  const bool fdx = fi > 0 && fi < P;
  const float fx = intr[0], fy = intr[1], cx = intr[2], cy = intr[3];
  const int g0 = w.gptr[s], g1 = w.gptr[s + 1];
  __shared__ float tab[kEtab];
  __shared__ float uvec[6];
  int pix[kLinPPT];
  float dsp[kLinPPT], xn[kLinPPT], yn[kLinPPT], acc[kLinPPT];
#pragma unroll
  for (int k = 0; k < kLinPPT; ++k) {
    pix[k] = blockIdx.y * kLinChunk + k * kLinThreads + threadIdx.x;
    const int pc = pix[k] < HW ? pix[k] : HW - 1;
    dsp[k] = disps[(int64_t)f * HW + pc];
    const int vi = pc / wd;
    xn[k] = ((float)(pc - vi * wd) - cx) / fx;
    yn[k] = ((float)vi - cy) / fy;
    acc[k] = 0.f;
  }
  for (int g = g0; g < g1; ++g) {
    const int e = w.gedge[g];
    __syncthreads();
    if (threadIdx.x < kEtab) tab[threadIdx.x] = w.etab[(int64_t)e * kEtab + threadIdx.x];
    if (threadIdx.x < 6) {
      const int j = (int)(jj[e] - t0);
      float u = (j > 0 && j < P) ? dx[j * 6 + threadIdx.x] : 0.f;
      if (fdx) {
        const float* L = w.etab + (int64_t)e * kEtab + 8;
#pragma unroll
        for (int r = 0; r < 6; ++r) u += L[r * 6 + threadIdx.x] * dx[fi * 6 + r];
      }
      uvec[threadIdx.x] = u;
    }
    __syncthreads();
    if (jj[e] == f) continue;   // self edge: E_j = 0
    const float* wgt = weights + (int64_t)e * 2 * HW;
#pragma unroll
    for (int k = 0; k < kLinPPT; ++k) {
      const int p = pix[k];
      if (p >= HW) continue;
      float H[32], cs = 0.f, ws = 0.f, Ej[6];
#pragma unroll
      for (int i = 0; i < 32; ++i) H[i] = 0.f;
      lin_pixel(tab, fx, fy, cx, cy, xn[k], yn[k], dsp[k], 0.f, 0.f, wgt[p], wgt[HW + p], false, H, cs, ws, Ej);
      float d = 0.f;
#pragma unroll
      for (int r = 0; r < 6; ++r) d = fmaf(Ej[r], uvec[r], d);
      acc[k] += d;
    }
  }
#pragma unroll
  for (int k = 0; k < kLinPPT; ++k) {
    const int p = pix[k];
    if (p >= HW) continue;
    const int64_t o = (int64_t)s * HW + p;
    const float v = w.qbuf[o] * (w.wbuf[o] - acc[k]);
    dz[o] = v;
    disps[(int64_t)f * HW + p] += v;
  }
}

// Tensor map over the E planes [6*rows, HW] (row stride row_stride(HW) floats): boxes of
// 64 plane rows x 32 pixels, 128B swizzle, zero fill past HW.
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static int encode_erows_map(CUtensorMap* map, float* erows, int HW, int64_t plane_rows) {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    cudaDriverEntryPointQueryResult q;
    void* f = nullptr;
    HS2_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q));
    if (q != cudaDriverEntryPointSuccess || !f) {
      set_error("cuTensorMapEncodeTiled is not available from the driver");
      return HS2_ERR_CUDA;
    }
    fn = reinterpret_cast<EncodeTiledFn>(f);
  }
  const cuuint64_t dims[2] = {(cuuint64_t)HW, (cuuint64_t)plane_rows};
  const cuuint64_t strides[1] = {(cuuint64_t)row_stride(HW) * sizeof(float)};
  const cuuint32_t box[2] = {(cuuint32_t)kTcK, (cuuint32_t)kTcBox};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, erows, dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed (%d)", (int)r);
    return HS2_ERR_CUDA;
  }
  return HS2_OK;
}

// ------------------------------------------------------------- cholesky ---
// Damped FP64 Cholesky factorisation + solve of the reduced camera system in one
// cooperative (persistent) launch, one CTA per SM:
//
//   damping   diag += ep + lm*diag                                          | barrier
//   panel 0                                                                 | barrier
//   for kb = 0 .. nbk-2 (look-ahead by one panel)
//     A   column block kb+1 -= L[:, kb] L[kb+1, kb]^T in 16-row slices      | per-row counters
//     B   panel kb+1 on `rest` CTAs (each waits for its two block rows'
//         slices), in parallel with the remaining tiles of update kb
//         (column blocks kb+2 ..) on the other CTAs                         | barrier
//   backward  x_c = L_cc^-T (y_c - sum_{j>c} L_jc^T x_j), one CTA per block c,
//             ordered by per-block ready flags instead of grid barriers; L_cc^-1
//             formed in shared memory while the blocks above are solved
//
// Panel kb, task t: the CTA holds [D; X | b] in shared memory (D the 64x64 diagonal
// block, redundantly in every CTA of the panel; X the t-th 64-row tile below D, none
// for t == 0; b the right-hand side) and eliminates the 64 columns in four 16-column
// sub-panels, left-looking: (a) the sub-panel columns receive the updates of the
// sub-panels left of them, (b) one warp factors the 16x16 diagonal sub-block and
// its part of b in registers, exchanging columns by shuffles, (c) every row below
// solves its 16 entries against that sub-block.  Task 0 writes L11, the reciprocal
// pivots and y = L11^-1 b1; the others write L21 and b2 - L21 y1.
//
// A non-positive pivot is seen identically by every CTA that factors the panel; the
// solution is then 0, as in the reference's solver fallback.  Every spin (grid
// barrier, ready flag) is bounded: on timeout the kernel sets HS2_DEV_TIMEOUT and
// returns.  Data written inside the launch is read through L2 (ld.global.cg).
constexpr int kCholThreads = 256;
constexpr int kPLD = 66;   // padded row length (doubles) of panel/tile rows in shared memory
constexpr unsigned kBarrierSpins = 1u << 22;
constexpr int kCtlFlags = 4;   // ctl[4 + c]: x of block c is final
// A panel's X tile (the 64 rows of one block row below D) is split over kXSplit tasks of
// kXRows rows, so the tasks that carry the pivot chain are no longer than the D-only task
// by a whole tile's solve; each task counts itself on its block row.
constexpr int kXSplit = 2;
constexpr int kXRows = 64 / kXSplit;

struct CholBuf {
  double* L11;      // [nbk][64][64] factored diagonal blocks (zero above the diagonal)
  double* dinv;     // [nbk][64] reciprocals of their diagonals
  double* y;        // [n] forward-substituted right-hand side
  unsigned* ctl;    // [0] barrier count, [1] barrier generation, [2] failed, [4 + c] ready flags,
                    // [4 + nbk + R] phase-A slices done on block row R,
                    // [4 + 2 nbk + R] panels whose L of block row R is written,
                    // [4 + 3 nbk + R nbk + C] trailing (phase-B) updates applied to tile (R, C)
};

__device__ __forceinline__ double2 ldcg2(const double* p) {
  return __ldcg(reinterpret_cast<const double2*>(p));
}
__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_gpu(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed_gpu(unsigned* p, unsigned v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned atom_add_acq_rel_gpu(unsigned* p, unsigned v) {
  unsigned old;
  asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}

// Sense-free generation barrier over all CTAs of the cooperative launch.  The
// __syncthreads before thread 0's acq_rel arrival publishes the CTA's writes; the
// acquire of the new generation + __syncthreads makes the other CTAs' writes visible.
__device__ __forceinline__ bool grid_barrier(unsigned* ctl, unsigned nblocks, int32_t* info) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned gen = ld_acquire_gpu(ctl + 1);
    int ok = 1;
    if (atom_add_acq_rel_gpu(ctl, 1u) == nblocks - 1) {
      st_relaxed_gpu(ctl, 0u);
      st_release_gpu(ctl + 1, gen + 1);
    } else {
      unsigned spins = 0;
      while (ld_acquire_gpu(ctl + 1) == gen) {
        if (++spins > kBarrierSpins) {
          ok = 0;
          atomicOr(info, HS2_DEV_TIMEOUT);
          break;
        }
        if (spins > 64) __nanosleep(32);
      }
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

__device__ __forceinline__ void red_release_add_gpu(unsigned* p, unsigned v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Panel kb+1, task t reads block rows kb+1 (D) and kb+1+t (X) of column block kb+1: waits
// until the four phase-A slices of each have been applied for every panel up to kb.
__device__ bool chol_wait_slices(const unsigned* slices, int kb, int t, int32_t* info) {
  __shared__ int s_bad;
  if (threadIdx.x == 0) {
    const unsigned target = 4u * (unsigned)(kb + 1);
    int bad = 0;
    for (int k = 0; k < (t > 0 ? 2 : 1) && !bad; ++k) {
      const unsigned* c = slices + kb + 1 + (k ? t : 0);
      unsigned spins = 0;
      while (ld_acquire_gpu(c) < target) {
        if (++spins > kBarrierSpins) {
          atomicOr(info, HS2_DEV_TIMEOUT);
          bad = 1;
          break;
        }
        if (spins > 64) __nanosleep(32);
      }
    }
    s_bad = bad;
  }
  __syncthreads();
  return s_bad == 0;
}

// Waits (thread 0) until *c >= target; false on timeout, or at once when another wait of
// the launch has already timed out.
__device__ __forceinline__ bool wait_count(const unsigned* c, unsigned target, int32_t* info) {
  unsigned spins = 0;
  while (ld_acquire_gpu(c) < target) {
    if ((++spins & 255u) == 0 && (*(volatile int32_t*)info & HS2_DEV_TIMEOUT)) return false;
    if (spins > kBarrierSpins) {
      atomicOr(info, HS2_DEV_TIMEOUT);
      return false;
    }
    if (spins > 64) __nanosleep(32);
  }
  return true;
}

// A trailing-update task on tile (R, C) with panel kb: waits until panel kb has written
// the L blocks of rows R and C and the tile holds the phase-B updates of panels < kb
// (tcnt >= tdone).  CTA-wide result.
__device__ bool chol_wait_tile(const unsigned* lcnt, const unsigned* tcnt, int nbk, int kb, int R, int C,
                               unsigned tdone, int32_t* info) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0)
    s_ok = wait_count(lcnt + R, kXSplit * (kb + 1), info) && wait_count(lcnt + C, kXSplit * (kb + 1), info) &&
           wait_count(tcnt + (int64_t)R * nbk + C, tdone, info);
  __syncthreads();
  return s_ok != 0;
}

// Waits (thread 0) until the ready flag is set; false on timeout.
__device__ __forceinline__ bool wait_flag(const unsigned* f, int32_t* info) {
  unsigned spins = 0;
  while (ld_acquire_gpu(f) == 0u) {
    if (++spins > kBarrierSpins) {
      atomicOr(info, HS2_DEV_TIMEOUT);
      return false;
    }
    if (spins > 64) __nanosleep(32);
  }
  return true;
}

// d(8x8, two values per lane) += a(8x4) b(4x8) in FP64 on the tensor cores (mma.sync
// m8n8k4): lane l holds a[l/4][l%4], b[l%4][l/4] and d[l/4][2(l%4) + {0,1}].
__device__ __forceinline__ void dmma_m8n8k4(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d0), "+d"(d1) : "d"(a), "d"(b));
}

// (b) One warp factors the nsb x nsb diagonal sub-block at (c0, c0) in registers,
// fraction-free with 2 x 2 pivot blocks: with u, v the trailing columns j, j+1, the block
// P = [p q; q s] and det = p s - q^2, step (j, j+1) replaces the trailing entries by
//   (A_rk det - [u_r v_r] adj(P) [u_k v_k]^T) 2^-E,   E the binary exponent of det,
// so no reciprocal sits on the chain from one pivot block to the next and the exact
// power-of-two scale keeps the entries in range.  The trailing block is then c times the
// true Schur complement, c <- c det 2^-E.  Eliminating column j alone would give the
// scale c p and column j+1 the entries w_r = p v_r - q u_r with pivot det, so with
// cd = (c p, c p det) and f = (c, c p) for the two columns:
//   L_rk = num_rk / sqrt(cd_k),   1/L_kk = f_k / sqrt(cd_k),   y_k = b'_k / sqrt(cd_k),
// num = u_r resp. w_r and b' = b_j resp. p b_j+1 - q b_j.  The products are recorded per
// column and L is formed after the loop, off the elimination chain.  Lane = row (0..15)
// + 16 * column half; a lane holds the 8 entries of its row in its half, padded with the
// identity outside nsb.  Columns j, j+1 (and b_j, b_j+1) are exchanged through a double-
// buffered 2 x 36 shared array, one __syncwarp per block step.  Writes L (lower part),
// the multipliers M_rj = L_rj / L_jj above the diagonal (row j), 1/L_jj to sv and y to bv.
__device__ __forceinline__ void chol_factor_diag(double (*Pm)[kPLD], double* bv, double* sv, double* xc, int c0,
                                                 int nsb, int* sfail) {
  const int lane = threadIdx.x & 31, rr = lane & 15, hh = lane >> 4;
  double a[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const int k = 8 * hh + q;
    a[q] = (rr < nsb && k < nsb) ? Pm[c0 + rr][c0 + k] : (rr == k ? 1.0 : 0.0);
  }
  double bb = (hh == 0 && rr < nsb) ? bv[c0 + rr] : 0.0;
  double cfac = 1.0;
  // per own column k = 8 hh + q: cd_k and f_k; for the own row: cd, f and b' at its step
  double cq[8], fq[8], my_cd = 1.0, my_f = 1.0, my_b = 0.0;
#pragma unroll
  for (int q = 0; q < 8; ++q) cq[q] = fq[q] = 1.0;
  bool ok = true;
#pragma unroll
  for (int j = 0; j < 16; j += 2) {
    const int hj = j >> 3, qj = j & 7;
    double* col = xc + ((j >> 1) & 1) * 36;   // [0,16) u, [16,32) v, [32] b_j, [33] b_j+1
    if (hh == hj) {
      col[rr] = a[qj];
      col[16 + rr] = a[qj + 1];
    }
    if (lane == j || lane == j + 1) col[32 + lane - j] = bb;
    __syncwarp();
    const double p = col[j], q = col[j + 1], s = col[16 + j + 1];
    const double ur = col[rr], vr = col[16 + rr];
    const double2 bjj = *reinterpret_cast<const double2*>(&col[32]);
    double uk[8], vk[8];
#pragma unroll
    for (int t = 0; t < 8; t += 2) {
      const double2 x = *reinterpret_cast<const double2*>(&col[8 * hh + t]);
      const double2 y = *reinterpret_cast<const double2*>(&col[16 + 8 * hh + t]);
      uk[t] = x.x;
      uk[t + 1] = x.y;
      vk[t] = y.x;
      vk[t + 1] = y.y;
    }
    const double det = fma(p, s, -(q * q));
    ok = ok && (p > 0.0) && (det > 0.0);
    const long long bits = __double_as_longlong(det);
    const double sc = __longlong_as_double((2046LL - ((bits >> 52) & 0x7FF)) << 52);   // 2^-E
    const double w1 = fma(s, ur, -(q * vr)), w2 = fma(p, vr, -(q * ur));
    const double dets = det * sc, w1s = w1 * sc, w2s = w2 * sc;
#pragma unroll
    for (int t = 0; t < 8; ++t)
      if (8 * hh + t > j + 1) a[t] = fma(a[t], dets, -fma(w1s, uk[t], w2s * vk[t]));
    const double bj1 = fma(p, bjj.y, -(q * bjj.x));
    if (hh == 0 && rr > j + 1) bb = fma(bb, dets, -fma(w1s, bjj.x, w2s * bjj.y));
    // columns j, j+1 are final: only registers are written here
    const double cp = cfac * p, cpd = cp * det;
    if (hh == hj) {
      a[qj + 1] = w2;
      cq[qj] = cp;
      fq[qj] = cfac;
      cq[qj + 1] = cpd;
      fq[qj + 1] = cp;
    }
    if (rr == j) {
      my_cd = cp;
      my_f = cfac;
      my_b = bjj.x;
    }
    if (rr == j + 1) {
      my_cd = cpd;
      my_f = cp;
      my_b = bj1;
    }
    cfac *= dets;
  }
  if (rr < nsb) {
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int k = 8 * hh + q;
      if (k <= rr) {
        const double s = rsqrt(cq[q]);
        const double l = a[q] * s;
        Pm[c0 + rr][c0 + k] = l;
        if (k < rr) Pm[c0 + k][c0 + rr] = l * (fq[q] * s);
      }
    }
    if (hh == 0) {
      const double s = rsqrt(my_cd);
      sv[c0 + rr] = my_f * s;
      bv[c0 + rr] = my_b * s;
    }
  }
  if (lane == 0 && !ok) *sfail = 1;
}

// Panel kb, task t (0: D only; t >= 1: D and the (t-1)-th tile below it).  Returns
// false when a pivot is not positive (ctl[2] is then set).
__device__ bool chol_panel(int n, int kb, int t, int xh, double* __restrict__ A, double* __restrict__ bvec,
                           CholBuf cb, double* csm) {
  const int tid = threadIdx.x;
  const int o = kb * kNB, nb = min(kNB, n - o);
  const int r0 = o + nb + (t - 1) * kNB + xh * kXRows;
  const int nr = t == 0 ? 0 : max(0, min(kXRows, n - r0));
  double (*Pm)[kPLD] = reinterpret_cast<double (*)[kPLD]>(csm);   // [128][kPLD]: D rows, then X rows
  double* bv = csm + 128 * kPLD;                                   // [128]
  double* sv = bv + 128;                                           // [64] 1/L_jj
  double* xc = sv + 64;                                            // [72] column exchange of (b)
  int* sfail = reinterpret_cast<int*>(xc + 72);
  __syncthreads();
#pragma unroll
  for (int half = 0; half < 2; ++half) {
    double2 v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int idx = tid + (half * 8 + q) * kCholThreads;   // double2 index in the 128 x 32 grid
      const int r = idx >> 5, k = (idx & 31) * 2;
      const bool live = r < kNB ? r < nb : r - kNB < nr;
      const double* src = A + (int64_t)(r < kNB ? o + r : r0 + r - kNB) * n + o + k;
      v[q] = make_double2(0.0, 0.0);
      if (live && k + 1 < nb) v[q] = ldcg2(src);   // n is even: a pair never leaves the row
      else if (live && k < nb) v[q].x = __ldcg(src);
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int idx = tid + (half * 8 + q) * kCholThreads;
      *reinterpret_cast<double2*>(&Pm[idx >> 5][(idx & 31) * 2]) = v[q];
    }
  }
  if (tid < 128) {
    const int r = tid;
    bv[r] = r < kNB ? (r < nb ? __ldcg(&bvec[o + r]) : 0.0) : (r - kNB < nr ? __ldcg(&bvec[r0 + r - kNB]) : 0.0);
  }
  if (tid == 0) *sfail = 0;
  __syncthreads();
  for (int c0 = 0; c0 < nb; c0 += 16) {
    const int c1 = min(c0 + 16, nb);
    if (c0 > 0) {
      const int lane = tid & 31, warp = tid >> 5;
      // (a) left-looking update of the sub-panel columns [c0, c0+16) of the rows >= c0 and the
      // X rows by FP64 tensor-core MMA (m8n8k4): a warp owns an 8-row tile and both 8-column
      // halves, k runs over the c0 columns already eliminated.
      const int td = (((nb + 7) >> 3) - (c0 >> 3)), tx = (nr + 7) >> 3;
      for (int tile = warp; tile < td + tx; tile += kCholThreads / 32) {
        const int rt = tile < td ? c0 + 8 * tile : kNB + 8 * (tile - td);
        double d00 = 0.0, d01 = 0.0, d10 = 0.0, d11 = 0.0;
        for (int k0 = 0; k0 < c0; k0 += 4) {
          const double av = Pm[rt + (lane >> 2)][k0 + (lane & 3)];
          const double b0 = Pm[c0 + (lane >> 2)][k0 + (lane & 3)];
          const double b1 = Pm[c0 + 8 + (lane >> 2)][k0 + (lane & 3)];
          dmma_m8n8k4(d00, d01, av, b0);
          dmma_m8n8k4(d10, d11, av, b1);
        }
        double* row = Pm[rt + (lane >> 2)] + c0 + (lane & 3) * 2;
        row[0] -= d00;
        row[1] -= d01;
        row[8] -= d10;
        row[9] -= d11;
      }
      if (tid < c1 - c0) {
        const int r = c0 + tid;
        double b0 = 0.0, b1 = 0.0;
        for (int k = 0; k < c0; k += 2) {
          b0 = fma(Pm[r][k], bv[k], b0);
          b1 = fma(Pm[r][k + 1], bv[k + 1], b1);
        }
        bv[r] -= b0 + b1;
      }
      __syncthreads();
    }
    // (b)
    if (tid < 32) chol_factor_diag(Pm, bv, sv, xc, c0, c1 - c0, sfail);
    __syncthreads();
    if (*sfail) {
      if (tid == 0) atomicExch(cb.ctl + 2, 1u);
      return false;
    }
    // (c) rows below the sub-block solve x L_ss^T = v: with u_j = x_j L_jj,
    // u_j = v_j - sum_{i<j} u_i M_ji (M above the diagonal of the sub-block), x = u / L_jj
    if (tid < 128) {
      const int r = tid;
      if (r >= kNB ? (r - kNB < nr) : (r >= c1 && r < nb)) {
        double v[16];
#pragma unroll
        for (int l = 0; l < 16; ++l) v[l] = c0 + l < c1 ? Pm[r][c0 + l] : 0.0;
#pragma unroll
        for (int j = 0; j < 15; ++j) {
          if (c0 + j < c1) {
#pragma unroll
            for (int l = (j + 1) & ~1; l < 16; l += 2) {
              const double2 m = *reinterpret_cast<const double2*>(&Pm[c0 + j][c0 + l]);
              if (l > j) v[l] = fma(-v[j], m.x, v[l]);
              v[l + 1] = fma(-v[j], m.y, v[l + 1]);
            }
          }
        }
#pragma unroll
        for (int l = 0; l < 16; ++l)
          if (c0 + l < c1) Pm[r][c0 + l] = v[l] * sv[c0 + l];
      }
    }
    __syncthreads();
  }
  // X rows: b2 -= L21 y1 (four threads per row)
  {
    const int i = tid >> 2, part = tid & 3;
    double s = 0.0;
    if (i < nr)
      for (int k = part; k < nb; k += 4) s = fma(Pm[kNB + i][k], bv[k], s);
    s += __shfl_xor_sync(0xffffffffu, s, 1);
    s += __shfl_xor_sync(0xffffffffu, s, 2);
    __syncthreads();
    if (i < nr && part == 0) bv[kNB + i] -= s;
  }
  __syncthreads();
  if (t == 0) {
    for (int idx = tid; idx < kNB * kNB; idx += kCholThreads) {
      const int i = idx >> 6, l = idx & 63;
      cb.L11[((int64_t)kb * kNB + i) * kNB + l] = (l <= i && i < nb) ? Pm[i][l] : 0.0;
    }
    if (tid < kNB) {
      cb.dinv[(int64_t)kb * kNB + tid] = tid < nb ? sv[tid] : 0.0;
      if (tid < nb) cb.y[o + tid] = bv[tid];
    }
  } else {
    for (int idx = tid; idx < nr * (kNB / 2); idx += kCholThreads) {
      const int i = idx >> 5, k = (idx & 31) * 2;
      double* dst = A + (int64_t)(r0 + i) * n + o + k;
      if (k + 1 < nb) *reinterpret_cast<double2*>(dst) = *reinterpret_cast<const double2*>(&Pm[kNB + i][k]);
      else if (k < nb) *dst = Pm[kNB + i][k];
    }
    if (tid < nr) bvec[r0 + tid] = bv[kNB + tid];
  }
  return true;
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, uint32_t src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

// A[ri + i][rj + j] -= sum_k L[ri + i][o + k] L[rj + j][o + k] over the 16*RG rows
// at ri and the 64 columns at rj; `diag` keeps only entries on or below the
// diagonal of A.  Thread (ty, tx) owns rows ty + 16a and columns tx + 16c.  Both L row
// blocks and the target tile itself arrive by 16-byte cp.async copies issued together
// (one L2 round trip; rows and columns outside the matrix are zero-filled).
template <int RG>
__device__ void chol_update_tile(int n, double* __restrict__ A, int o, int ri, int rj, bool diag, double* csm) {
  const int tid = threadIdx.x, ty = tid >> 4, tx = tid & 15;
  const int ni = min(16 * RG, n - ri), nj = min(kNB, n - rj);
  if (ni <= 0) return;
  constexpr int kRows = 16 * RG;
  double (*Ai)[kPLD] = reinterpret_cast<double (*)[kPLD]>(csm);
  double (*Aj)[kPLD] = reinterpret_cast<double (*)[kPLD]>(csm + 64 * kPLD);
  double (*Cs)[kPLD] = reinterpret_cast<double (*)[kPLD]>(csm + 128 * kPLD);
  __syncthreads();
  {
    const uint32_t sb = smem_u32(csm);
    for (int idx = tid; idx < (2 * kRows + 64) * 32; idx += kCholThreads) {
      const int r = idx >> 5, k = (idx & 31) * 2;
      int srow, a;
      int64_t grow;
      int gcol;
      bool live;
      if (r < kRows) {                       // L rows of the tile's block rows
        srow = r;
        live = r < ni;
        grow = ri + r;
        gcol = o + k;
      } else if (r < kRows + 64) {           // L rows of the tile's block columns
        a = r - kRows;
        srow = 64 + a;
        live = a < nj;
        grow = rj + a;
        gcol = o + k;
      } else {                               // the tile
        a = r - kRows - 64;
        srow = 128 + a;
        live = a < ni && k < nj;
        grow = ri + a;
        gcol = rj + k;
      }
      cp_async16(sb + (uint32_t)(srow * kPLD + k) * 8u, live ? (const void*)(A + grow * n + gcol) : (const void*)A,
                 live ? 16u : 0u);
    }
    cp_async_wait_all();
  }
  __syncthreads();
  double acc[RG][4];
#pragma unroll
  for (int a = 0; a < RG; ++a)
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[a][c] = 0.0;
#pragma unroll 2
  for (int k = 0; k < kNB; k += 2) {
    double2 va[RG], vb[4];
#pragma unroll
    for (int a = 0; a < RG; ++a) va[a] = *reinterpret_cast<const double2*>(&Ai[ty + 16 * a][k]);
#pragma unroll
    for (int c = 0; c < 4; ++c) vb[c] = *reinterpret_cast<const double2*>(&Aj[tx + 16 * c][k]);
#pragma unroll
    for (int a = 0; a < RG; ++a)
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        acc[a][c] = fma(va[a].x, vb[c].x, acc[a][c]);
        acc[a][c] = fma(va[a].y, vb[c].y, acc[a][c]);
      }
  }
#pragma unroll
  for (int a = 0; a < RG; ++a)
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int i = ty + 16 * a, j = tx + 16 * c;
      if (i < ni && j < nj && (!diag || rj + j <= ri + i)) A[(int64_t)(ri + i) * n + rj + j] = Cs[i][j] - acc[a][c];
    }
}

// Backward substitution L^T x = y, block c on CTA c mod G (blocks taken from the
// highest down).  The CTA first inverts L_cc in shared memory (row by row,
// X_ij = -(1/L_ii) sum_{k=j}^{i-1} L_ik X_kj, column j on four threads each summing every
// fourth k) -- for every block but the highest this overlaps the wait for the blocks
// above -- then folds L_jc^T x_j into per-thread partial sums as the ready flags of
// blocks j > c arrive (its loads of L_jc are issued before it waits), and forms
// x_c = L_cc^-T (y_c - sum_j L_jc^T x_j) as one mat-vec: no 64-step dependency chain
// sits between two ready flags.
__device__ bool chol_backward(int n, int nbk, const double* __restrict__ A, CholBuf cb, double* __restrict__ x,
                              float* __restrict__ dx_out, int32_t* __restrict__ info, double* csm) {
  const int tid = threadIdx.x;
  const int G = (int)gridDim.x, cta = (int)blockIdx.x;
  if (cta >= nbk) return true;
  constexpr unsigned kFull = 0xffffffffu;
  double (*Ls)[kNB] = reinterpret_cast<double (*)[kNB]>(csm);              // [64][64] L_cc
  double (*Li)[kNB] = reinterpret_cast<double (*)[kNB]>(csm + kNB * kNB);  // [64][64] L_cc^-1
  double* ys = csm + 2 * kNB * kNB;                                         // [64]
  double* dv = ys + kNB;                                                    // [64] 1/L_ii
  double* part = dv + kNB;                                                  // [4][64]
  double* rv = part + 4 * kNB;                                              // [64]
  __shared__ int s_abort;
  const int cl = tid & 63, rg = tid >> 6;
  const int ic = tid >> 2, is = tid & 3;   // inversion: column ic, k phase is
  for (int c = cta + ((nbk - 1 - cta) / G) * G; c >= 0; c -= G) {
    const int oc = c * kNB, nc = min(kNB, n - oc);
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int idx = tid + q * kCholThreads;
      *reinterpret_cast<double2*>(&Ls[idx >> 5][(idx & 31) * 2]) =
          ldcg2(&cb.L11[((int64_t)c * kNB + (idx >> 5)) * kNB + (idx & 31) * 2]);
    }
    if (tid < kNB) {
      ys[tid] = tid < nc ? __ldcg(&cb.y[oc + tid]) : 0.0;
      dv[tid] = tid < nc ? __ldcg(&cb.dinv[(int64_t)c * kNB + tid]) : 0.0;
    }
    __syncthreads();
    for (int idx = tid; idx < kNB * kNB; idx += kCholThreads) {
      const int i = idx >> 6, l = idx & 63;
      Li[i][l] = i == l ? dv[i] : 0.0;
    }
    __syncthreads();
    for (int i = 1; i < nc; ++i) {
      double p0 = 0.0, p1 = 0.0;
      if (ic < i) {
        int k = ic + is;
        for (; k + 4 < i; k += 8) {
          p0 = fma(Ls[i][k], Li[k][ic], p0);
          p1 = fma(Ls[i][k + 4], Li[k + 4][ic], p1);
        }
        if (k < i) p0 = fma(Ls[i][k], Li[k][ic], p0);
      }
      double pv = p0 + p1;
      pv += __shfl_xor_sync(kFull, pv, 1);
      pv += __shfl_xor_sync(kFull, pv, 2);
      if (ic < i && is == 0) Li[i][ic] = -dv[i] * pv;
      __syncthreads();
    }
    double acc = 0.0;
    for (int j = nbk - 1; j > c; --j) {
      const int oj = j * kNB, nj = min(kNB, n - oj);
      double lv[16];
#pragma unroll
      for (int r = 0; r < 16; ++r) {
        const int row = rg * 16 + r;
        lv[r] = (row < nj && cl < nc) ? __ldcg(&A[(int64_t)(oj + row) * n + oc + cl]) : 0.0;
      }
      if (tid == 0) s_abort = wait_flag(cb.ctl + kCtlFlags + j, info) ? 0 : 1;
      __syncthreads();
      if (s_abort) return false;
#pragma unroll
      for (int r = 0; r < 16; ++r) {
        const int row = rg * 16 + r;
        const double xv = row < nj ? __ldcg(&x[oj + row]) : 0.0;
        acc = fma(lv[r], xv, acc);
      }
    }
    part[rg * kNB + cl] = acc;
    __syncthreads();
    if (tid < kNB) rv[tid] = ys[tid] - ((part[tid] + part[kNB + tid]) + (part[2 * kNB + tid] + part[3 * kNB + tid]));
    __syncthreads();
    // x_i = sum_{k >= i} Li[k][i] r_k: output cl, rows k of quarter rg
    {
      double v = 0.0;
#pragma unroll
      for (int r = 0; r < 16; ++r) {
        const int k = rg * 16 + r;
        if (k >= cl) v = fma(Li[k][cl], rv[k], v);
      }
      part[rg * kNB + cl] = v;
    }
    __syncthreads();
    if (tid < nc) {
      const double xv = (part[tid] + part[kNB + tid]) + (part[2 * kNB + tid] + part[3 * kNB + tid]);
      x[oc + tid] = xv;
      dx_out[oc + tid] = (float)xv;
    }
    __syncthreads();
    if (tid == 0) st_release_gpu(cb.ctl + kCtlFlags + c, 1u);
  }
  return true;
}

__global__ void __launch_bounds__(kCholThreads, 1)
ba_cholesky_kernel(int n, float lm, float ep, BaPtrs w, CholBuf cb, float* __restrict__ dx_out,
                   int32_t* __restrict__ info) {
  if (info[0]) return;
  extern __shared__ __align__(16) double csm[];
  const unsigned G = gridDim.x;
  const int tid = threadIdx.x;
  const int nbk = (n + kNB - 1) / kNB;
  double* A = w.A;
  double* bvec = w.b;

  for (int i = blockIdx.x * kCholThreads + tid; i < n; i += G * kCholThreads) {
    double* d = &A[(int64_t)i * n + i];
    *d += (double)ep + (double)lm * __ldcg(d);
  }
  if (!grid_barrier(cb.ctl, G, info)) return;

  // Dataflow instead of a grid barrier per panel: every task waits (acquire) only for the
  // tasks that write its inputs and counts itself (release) when done.  A task of stage
  // A(kb) / B(kb) depends only on tasks of earlier stages and every CTA runs its tasks in
  // stage order, so with all CTAs resident (cooperative launch) no wait can cycle.  A
  // failed factorisation does not stop the schedule (results are discarded at the end).
  unsigned* slices = cb.ctl + kCtlFlags + nbk;
  unsigned* lcnt = cb.ctl + kCtlFlags + 2 * nbk;
  unsigned* tcnt = cb.ctl + kCtlFlags + 3 * nbk;
  // panel task tau of a panel with `rest` block rows from its diagonal down: tau = 0 is D
  // alone, tau >= 1 is half (tau - 1) % kXSplit of block row 1 + (tau - 1) / kXSplit
  for (int tau = blockIdx.x; tau < 1 + kXSplit * (nbk - 1); tau += G) {
    const int t = tau == 0 ? 0 : 1 + (tau - 1) / kXSplit, xh = tau == 0 ? 0 : (tau - 1) % kXSplit;
    chol_panel(n, 0, t, xh, A, bvec, cb, csm);
    __syncthreads();
    if (threadIdx.x == 0 && t > 0) red_release_add_gpu(lcnt + t, 1u);
  }

  for (int kb = 0; kb + 1 < nbk; ++kb) {
    const int o = kb * kNB;
    const int rest = nbk - kb - 1;
    // A: column block kb+1, 16-row slices of the tiles below panel kb; each slice counts
    // itself on its block row, which the panel tasks of phase B wait for
    for (int t = blockIdx.x; t < rest * 4; t += G) {
      const int I = t >> 2, q = t & 3;
      if (!chol_wait_tile(lcnt, tcnt, nbk, kb, kb + 1 + I, kb + 1, (unsigned)kb, info)) return;
      chol_update_tile<1>(n, A, o, o + kNB + I * kNB + 16 * q, o + kNB, I == 0, csm);
      __syncthreads();
      if (threadIdx.x == 0) red_release_add_gpu(slices + kb + 1 + I, 1u);
    }
    // B: panel kb+1 (tasks 0..rest-1) || tiles (I, J), 1 <= J <= I < rest, of update kb.
    // The panel tasks sit on CTAs of their own (they are the longer tasks); the tiles go
    // round-robin over the remaining CTAs.  A panel task counts the L block it writes on
    // its block row; a tile counts the update it applied.
    const int ntiles = rest * (rest - 1) / 2;
    const int ntask = 1 + kXSplit * (rest - 1);
    const bool split = (int)G > ntask;
    const int tfirst = split ? ((int)blockIdx.x < ntask ? ntiles : (int)blockIdx.x - ntask) : (int)blockIdx.x;
    const int tstep = split ? (int)G - ntask : (int)G;
    auto panel_task = [&](int tau) -> bool {
      const int t = tau == 0 ? 0 : 1 + (tau - 1) / kXSplit, xh = tau == 0 ? 0 : (tau - 1) % kXSplit;
      if (!chol_wait_slices(slices, kb, t, info)) return false;
      chol_panel(n, kb + 1, t, xh, A, bvec, cb, csm);
      __syncthreads();
      if (threadIdx.x == 0 && t > 0) red_release_add_gpu(lcnt + kb + 1 + t, 1u);
      return true;
    };
    if (split && (int)blockIdx.x < ntask) {
      if (!panel_task(blockIdx.x)) return;
    }
    for (int t = tfirst; t < (split ? ntiles : ntask + ntiles); t += tstep) {
      if (!split && t < ntask) {
        if (!panel_task(t)) return;
        continue;
      }
      int I = 0, tt = split ? t : t - ntask;
      while (tt > I) {
        tt -= I + 1;
        ++I;
      }
      const int J = tt + 1;
      ++I;
      if (!chol_wait_tile(lcnt, tcnt, nbk, kb, kb + 1 + I, kb + 1 + J, (unsigned)kb, info)) return;
      chol_update_tile<4>(n, A, o, o + kNB + I * kNB, o + kNB + J * kNB, I == J, csm);
      __syncthreads();
      if (threadIdx.x == 0) red_release_add_gpu(tcnt + (int64_t)(kb + 1 + I) * nbk + kb + 1 + J, 1u);
    }
  }
  if (!grid_barrier(cb.ctl, G, info)) return;
  const bool failed = *(volatile unsigned*)(cb.ctl + 2) != 0;

  if (!failed) {
    chol_backward(n, nbk, A, cb, w.x, dx_out, info, csm);
    return;
  }
  for (int i = blockIdx.x * kCholThreads + tid; i < n; i += G * kCholThreads) {
    w.x[i] = 0.0;
    dx_out[i] = 0.0f;
  }
  if (blockIdx.x == 0 && tid == 0) atomicAdd(&info[2], 1);
}

// -------------------------------------------------------------- backsub ---
template <int NT, int PPT = kLinPPT>
__device__ __forceinline__ void ba_backsub_body(int s, int chunk, float* __restrict__ disps, int HW, int P, BaPtrs w,
                                                const float* __restrict__ dx, float* __restrict__ dz,
                                                int64_t dz_rows, const int32_t* __restrict__ info) {
  constexpr int kChunk = NT * PPT;
  if (info[0]) return;
  if (s >= info[1] || s >= dz_rows) return;
  const int f = w.kx[s];
  const int r0 = w.rptr[s], r1 = w.rptr[s + 1];
  const int HWs = row_stride(HW);
  constexpr int kRows = 64;                 // rows whose dx sit in shared memory at a time
  __shared__ float xs[kRows][6];
  float acc[PPT];
  int pix[PPT];
#pragma unroll
  for (int k = 0; k < PPT; ++k) {
    pix[k] = chunk * kChunk + k * NT + threadIdx.x;
    acc[k] = 0.f;
  }
  for (int rb = r0; rb < r1; rb += kRows) {
    const int nrw = min(kRows, r1 - rb);
    __syncthreads();
    for (int i = threadIdx.x; i < nrw * 6; i += NT) {
      const int ix = w.rpose[rb + i / 6];
      // reference EvT6x1_kernel skips rows of pose index <= 0
      xs[i / 6][i % 6] = (ix <= 0 || ix >= P) ? 0.f : dx[ix * 6 + i % 6];
    }
    __syncthreads();
#pragma unroll 8
    for (int i = 0; i < nrw; ++i) {
      const int ix = w.rpose[rb + i];
      if (ix <= 0 || ix >= P) continue;
      const float* Er = w.erows + ((int64_t)(rb + i) * 6) * HWs;
#pragma unroll
      for (int k = 0; k < PPT; ++k) {
        const int p = pix[k];
        if (p >= HW) continue;
        float d = 0.f;
#pragma unroll
        for (int c = 0; c < 6; ++c) d = fmaf(__ldcs(&Er[(int64_t)c * HWs + p]), xs[i][c], d);
        acc[k] += d;
      }
    }
  }
#pragma unroll
  for (int k = 0; k < PPT; ++k) {
    const int p = pix[k];
    if (p >= HW) continue;
    const int64_t o = (int64_t)s * HW + p;
    const float v = w.qbuf[o] * (w.wbuf[o] - acc[k]);
    dz[o] = v;
    disps[(int64_t)f * HW + p] += v;
  }
}

// 256 threads x 2 pixels over the linearisation's 512-pixel chunks (measured at 300 kf:
// 0.094 ms against 0.107 ms with 128 x 4)
constexpr int kBsThreads = 2 * kLinThreads;
constexpr int kBsPPT = kLinPPT / 2;
static_assert(kBsThreads * kBsPPT == kLinChunk, "back-substitution covers the linearisation's chunks");

__global__ void __launch_bounds__(kBsThreads)
ba_backsub_kernel(float* __restrict__ disps, int HW, int P, BaPtrs w, const float* __restrict__ dx,
                  float* __restrict__ dz, int64_t dz_rows, const int32_t* __restrict__ info) {
  ba_backsub_body<kBsThreads, kBsPPT>(blockIdx.x, blockIdx.y, disps, HW, P, w, dx, dz, dz_rows, info);
}

// ------------------------------------------------------------ pose retr ---
__device__ __forceinline__ void ba_pose_retr_body(int k, float* __restrict__ poses, int t0, int P, const BaPtrs w,
                                                  const int32_t* __restrict__ info) {
  if (info[0]) return;
  if (k >= P) return;
  float* p = poses + 7 * (int64_t)(t0 + k);
  double t[3] = {p[0], p[1], p[2]};
  double q[4] = {p[3], p[4], p[5], p[6]};
  double xi[6];
  for (int c = 0; c < 6; ++c) xi[c] = w.x[k * 6 + c];
  retract_left(xi, t, q);
  for (int c = 0; c < 3; ++c) p[c] = (float)t[c];
  for (int c = 0; c < 4; ++c) p[3 + c] = (float)q[c];
}

__global__ void ba_pose_retr_kernel(float* __restrict__ poses, int t0, int P, const BaPtrs w,
                                    const int32_t* __restrict__ info) {
  ba_pose_retr_body(blockIdx.x * blockDim.x + threadIdx.x, poses, t0, P, w, info);
}

// ------------------------------------------------------------ host side ---
struct BaProblem {
  int64_t num_poses, num_disps, K, E;
  int ht, wd, HW, t0, t1, P, motion_only;
};

static int ba_check(const BaProblem& p, const char* op) {
  if (p.ht <= 0 || p.wd <= 0 || p.E < 0 || p.num_poses <= 0 || p.num_disps <= 0) {
    set_error("%s: bad sizes (ht=%d wd=%d edges=%lld poses=%lld disps=%lld)", op, p.ht, p.wd,
              (long long)p.E, (long long)p.num_poses, (long long)p.num_disps);
    return HS2_ERR_INVALID;
  }
  if (p.t0 < 0 || p.t1 < p.t0 || p.t1 > p.K) {
    set_error("%s: need 0 <= t0 <= t1 <= min(num_poses, num_disps) (t0=%d t1=%d, frames=%lld)", op, p.t0,
              p.t1, (long long)p.K);
    return HS2_ERR_INVALID;
  }
  if (p.E > (1 << 24) || p.K > (1 << 24) || (int64_t)p.HW * 6 * (p.P + p.E) > ((int64_t)1 << 40)) {
    set_error("%s: problem too large", op);
    return HS2_ERR_INVALID;
  }
  return HS2_OK;
}

static BaProblem make_problem(int64_t num_poses, int64_t num_disps, int ht, int wd, int64_t E, int t0, int t1,
                              int motion_only) {
  BaProblem p;
  p.num_poses = num_poses;
  p.num_disps = num_disps;
  p.K = std::min(num_poses, num_disps);
  p.E = E;
  p.ht = ht;
  p.wd = wd;
  p.HW = ht * wd;
  p.t0 = t0;
  p.t1 = t1;
  p.P = t1 - t0;
  p.motion_only = motion_only ? 1 : 0;
  return p;
}

static int run_keys(const BaProblem& pb, const int64_t* ii, const int64_t* jj, int64_t eta_rows, BaPtrs w,
                    int32_t* info, cudaStream_t s) {
  HS2_CUDA(cudaMemsetAsync(info, 0, 4 * sizeof(int32_t), s));
  HS2_PROF("ba_keys", s);
  ba_keys_kernel<<<1, 1024, 0, s>>>(ii, jj, (int)pb.E, (int)pb.K, pb.t0, pb.t1, eta_rows, w, info);
  HS2_LAUNCH_CHECK("ba_keys_kernel");
  return HS2_OK;
}

static int run_cholesky(int n, float lm, float ep, BaPtrs w, CholBuf cb, float* dx, int32_t* info,
                        cudaStream_t s) {
  if (n == 0) return HS2_OK;
  HS2_PROF("ba_cholesky", s);
  const int nbk = (n + kNB - 1) / kNB;
  // panel: [128][kPLD] + b, 1/L_jj, exchange; tile: [192][kPLD]; backward: 2 x 64 x 64 + 256
  const size_t smem = sizeof(double) * std::max<size_t>(128 * kPLD + 128 + 64 + 72 + 2, 192 * kPLD);
  static DeviceOnce once;
  static std::atomic<int> grid_cap[kMaxDevices];
  int dev = 0;
  HS2_CUDA(cudaGetDevice(&dev));
  int rc = once.run(dev, [&]() -> int {
    int sms = 0, occ = 0;
    HS2_CUDA(cudaFuncSetAttribute(ba_cholesky_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    HS2_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    HS2_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, ba_cholesky_kernel, kCholThreads, smem));
    grid_cap[dev].store(std::max(1, std::min(occ, 1) * sms), std::memory_order_relaxed);
    return HS2_OK;
  });
  if (rc) return rc;
  const int work = std::max(std::max(nbk, (nbk - 1) * nbk / 2), (n + kCholThreads - 1) / kCholThreads);
  int G = std::max(1, std::min(grid_cap[dev].load(std::memory_order_relaxed), work));
  HS2_CUDA(cudaMemsetAsync(cb.ctl, 0, (kCtlFlags + 3 * (size_t)nbk + (size_t)nbk * nbk) * sizeof(unsigned), s));
  void* args[] = {&n, &lm, &ep, &w, &cb, &dx, &info};
  HS2_CUDA(cudaLaunchCooperativeKernel((const void*)ba_cholesky_kernel, dim3(G), dim3(kCholThreads), args, smem, s));
  HS2_LAUNCH_CHECK("ba_cholesky_kernel");
  return HS2_OK;
}

struct BaLaunch {
  int nchunk, schur_split, schur_chunk, tc_split, tc_chunk, f_split, f_chunk;
};

// Linearisation / Schur Gram path:
//   0  unfused linearisation writing the E rows, tcgen05 Gram over the stored rows
//      (SIMT above kTcMaxBlocks rows);
//   1  unfused linearisation, SIMT FP32 Gram for every frame;
//   2  fused per-frame kernel (E rows stay in shared memory, tcgen05 3xTF32 Gram) for
//      frames of at most kFMaxEdges edges and kFMaxRows Schur rows, the unfused
//      linearisation + SIMT Gram for the others, back-substitution recomputing E.
static std::atomic<int> g_schur_path{0};
// Precision of the tensor-core Gram: 1 = 3xTF32 (hi.hi + hi.lo + lo.hi, FP32-accurate,
// the default), 0 = one TF32 product (the reduced-precision Hessian of the mixed form).
static std::atomic<int> g_gram_split3{1};

static BaLaunch ba_launch_shape(const BaProblem& p) {
  BaLaunch l;
  const int64_t S = std::min<int64_t>(p.K, (int64_t)p.P + p.E);
  l.nchunk = (p.HW + kLinChunk - 1) / kLinChunk;
  // Schur split: about 8 waves of CTAs (2 resident per SM), chunks of >= 128 pixels
  l.schur_split = (int)std::max<int64_t>(1, std::min<int64_t>(std::max(1, p.HW / 128),
                                                              (16 * kNumSMs + S - 1) / std::max<int64_t>(S, 1)));
  l.schur_chunk = (p.HW + l.schur_split - 1) / l.schur_split;
  l.schur_chunk = (l.schur_chunk + kSchurTP - 1) / kSchurTP * kSchurTP;
  l.schur_split = (p.HW + l.schur_chunk - 1) / l.schur_chunk;
  // tensor-core split: about 4 waves of one-CTA-per-SM work units, >= 64 pixels each
  l.tc_split = (int)std::max<int64_t>(1, std::min<int64_t>(std::max(1, p.HW / 64),
                                                           (4 * kNumSMs + S - 1) / std::max<int64_t>(S, 1)));
  l.tc_chunk = (p.HW + l.tc_split - 1) / l.tc_split;
  l.tc_chunk = (l.tc_chunk + kTcK - 1) / kTcK * kTcK;
  l.tc_split = (p.HW + l.tc_chunk - 1) / l.tc_chunk;
  // fused split: about 3 waves of one-CTA-per-SM work units, >= 4 chunks of kFK pixels each
  const int fch = (p.HW + kFK - 1) / kFK;
  l.f_split = (int)std::max<int64_t>(1, std::min<int64_t>(std::max(1, fch / 4),
                                                          (3 * kNumSMs + S - 1) / std::max<int64_t>(S, 1)));
  l.f_chunk = (fch + l.f_split - 1) / l.f_split * kFK;
  l.f_split = (p.HW + l.f_chunk - 1) / l.f_chunk;
  return l;
}

// Linearisation + assembly of the damped-to-be reduced camera system (A - S, b - v)
// for the current poses/disparities; Q, w and the E rows are left in the workspace.
static int build_system(const BaProblem& p, const BaLaunch& l, const float* poses, const float* disps,
                        const float* intrinsics, const float* targets, const float* weights, const float* eta,
                        int64_t eta_rows, const int64_t* ii, const int64_t* jj, BaPtrs w, int32_t* info,
                        cudaStream_t s) {
  const int E = (int)p.E;
  const int P = p.P;
  const int n = 6 * P;
  const int64_t S = std::min<int64_t>(p.K, (int64_t)P + E);
  if (E > 0) {
    HS2_PROF("ba_edge_setup", s);
    ba_edge_setup_kernel<<<(6 * E + 127) / 128, 128, 0, s>>>(poses, ii, jj, E, w.etab, w.etab64, info);
    HS2_LAUNCH_CHECK("ba_edge_setup_kernel");
    HS2_CUDA(cudaMemsetAsync(w.hedge, 0, sizeof(double) * 27 * (size_t)E, s));
  }
  if (n > 0) {
    HS2_PROF("ba_zero_system", s);
    HS2_CUDA(cudaMemsetAsync(w.A, 0, sizeof(double) * (size_t)n * n, s));
    HS2_CUDA(cudaMemsetAsync(w.b, 0, sizeof(double) * (size_t)n, s));
  }
  const int path = g_schur_path.load();
  const bool fused = !p.motion_only && path == 2;
  if (fused && S > 0) {
    static DeviceOnce once;
    int dev = 0;
    HS2_CUDA(cudaGetDevice(&dev));
    int rc = once.run(dev, [&]() -> int {
      HS2_CUDA(cudaFuncSetAttribute(ba_frame_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kFSmem));
      return HS2_OK;
    });
    if (rc) return rc;
    dim3 grid((unsigned)S, l.f_split);
    HS2_PROF("ba_frame", s);
    ba_frame_kernel<<<grid, kFThreads, kFSmem, s>>>(disps, p.HW, p.wd, intrinsics, targets, weights, eta, eta_rows,
                                                   jj, p.t0, p.t1, l.f_chunk, w, info);
    HS2_LAUNCH_CHECK("ba_frame_kernel");
  }
  if (S > 0) {
    dim3 grid((unsigned)S, l.nchunk);
    HS2_PROF("ba_linearize", s);
    ba_linearize_kernel<<<grid, kLinThreads, 0, s>>>(disps, p.HW, p.wd, intrinsics, targets, weights, eta,
                                                     eta_rows, jj, p.t0, p.t1, p.motion_only, fused ? 1 : 0, w,
                                                     info);
    HS2_LAUNCH_CHECK("ba_linearize_kernel");
  }
  if (E > 0 && n > 0) {
    HS2_PROF("ba_assemble", s);
    ba_assemble_kernel<<<(6 * E + 127) / 128, 128, 0, s>>>(ii, jj, E, p.t0, P, w, info);
    HS2_LAUNCH_CHECK("ba_assemble_kernel");
  }
  if (!p.motion_only && n > 0 && S > 0) {
    HS2_PROF("ba_schur", s);
    const bool simt_only = path != 0;
    if (!simt_only) {
      static DeviceOnce once;
      int dev = 0;
      HS2_CUDA(cudaGetDevice(&dev));
      int rc = once.run(dev, [&]() -> int {
        HS2_CUDA(cudaFuncSetAttribute(ba_schur_tc_kernel<6>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem));
        return HS2_OK;
      });
      if (rc) return rc;
      CUtensorMap emap;
      rc = encode_erows_map(&emap, w.erows, p.HW, 6 * ((int64_t)P + p.E));
      if (rc) return rc;
      dim3 grid((unsigned)S, 1u, l.tc_split);
      ba_schur_tc_kernel<6><<<grid, kTcThreads, kTcSmem, s>>>(emap, p.HW, l.tc_chunk, w, n, info,
                                                              g_gram_split3.load());
      HS2_LAUNCH_CHECK("ba_schur_tc_kernel");
    }
    dim3 grid((unsigned)S, l.schur_split);
    ba_schur_kernel<<<grid, 256, 0, s>>>(p.HW, l.schur_chunk, w, P, simt_only ? 1 : kTcMaxBlocks + 1,
                                         fused ? 1 : 0, info);
    HS2_LAUNCH_CHECK("ba_schur_kernel");
  }
  return HS2_OK;
}

}  // namespace hs2

extern "C" int hs2_ba_workspace_size(int64_t num_poses, int64_t num_disps, int ht, int wd, int64_t num_edges,
                                     int t0, int t1, int motion_only, size_t* bytes) {
  using namespace hs2;
  if (!bytes) {
    set_error("ba_workspace_size: null output");
    return HS2_ERR_INVALID;
  }
  BaProblem p = make_problem(num_poses, num_disps, ht, wd, num_edges, t0, t1, motion_only);
  int rc = ba_check(p, "ba_workspace_size");
  if (rc) return rc;
  *bytes = ba_layout(p.K, p.HW, p.E, p.P, p.motion_only).total;
  return HS2_OK;
}

extern "C" int hs2_ba_keys(int64_t num_poses, int64_t num_disps, int ht, int wd, const int64_t* ii,
                           const int64_t* jj, int64_t num_edges, int t0, int t1, int32_t* kx, int32_t* kk_exp,
                           int32_t* rows_ptr, int32_t* rows, int32_t* info, void* workspace,
                           size_t workspace_bytes, hs2_stream_t stream) {
  using namespace hs2;
  BaProblem p = make_problem(num_poses, num_disps, ht, wd, num_edges, t0, t1, 0);
  int rc = ba_check(p, "ba_keys");
  if (rc) return rc;
  const BaLayout L = ba_layout(p.K, p.HW, p.E, p.P, 0);
  if (!workspace || workspace_bytes < L.total) {
    set_error("ba_keys: workspace of %zu bytes required", L.total);
    return HS2_ERR_WORKSPACE;
  }
  if ((rc = bind_device(workspace))) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  BaPtrs w = ba_ptrs(workspace, L);
  if ((rc = run_keys(p, ii, jj, 1, w, info, s))) return rc;
  const int64_t R = p.P + p.E;
  const int64_t S = std::min<int64_t>(p.K, R);
  if (kx) HS2_CUDA(cudaMemcpyAsync(kx, w.kx, sizeof(int) * S, cudaMemcpyDeviceToDevice, s));
  if (rows_ptr) HS2_CUDA(cudaMemcpyAsync(rows_ptr, w.sptr, sizeof(int) * (S + 1), cudaMemcpyDeviceToDevice, s));
  if (rows) HS2_CUDA(cudaMemcpyAsync(rows, w.srow, sizeof(int) * R, cudaMemcpyDeviceToDevice, s));
  if (kk_exp && R > 0) {
    ba_kk_kernel<<<(unsigned)((R + 255) / 256), 256, 0, s>>>(ii, (int)p.E, p.t0, p.P, w.slot, kk_exp, info);
    HS2_LAUNCH_CHECK("ba_kk_kernel");
  }
  return HS2_OK;
}

extern "C" int hs2_ba(float* poses, int64_t num_poses, float* disps, int64_t num_disps, int ht, int wd,
                      const float* intrinsics, const float* targets, const float* weights, const float* eta,
                      int64_t eta_rows, const int64_t* ii, const int64_t* jj, int64_t num_edges, int t0, int t1,
                      int iterations, float lm, float ep, int motion_only, float* dx, float* dz, int64_t dz_rows,
                      int32_t* info, void* workspace, size_t workspace_bytes, hs2_stream_t stream) {
  using namespace hs2;
  BaProblem p = make_problem(num_poses, num_disps, ht, wd, num_edges, t0, t1, motion_only);
  int rc = ba_check(p, "ba");
  if (rc) return rc;
  if (iterations < 0) {
    set_error("ba: iterations must be >= 0");
    return HS2_ERR_INVALID;
  }
  if (!motion_only && eta_rows <= 0) {
    set_error("ba: eta must have at least one row");
    return HS2_ERR_INVALID;
  }
  const BaLayout L = ba_layout(p.K, p.HW, p.E, p.P, p.motion_only);
  if (!workspace || workspace_bytes < L.total) {
    set_error("ba: workspace of %zu bytes required (got %zu)", L.total, workspace_bytes);
    return HS2_ERR_WORKSPACE;
  }
  if ((rc = bind_device(poses))) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  BaPtrs w = ba_ptrs(workspace, L);
  if ((rc = run_keys(p, ii, jj, motion_only ? 1 : eta_rows, w, info, s))) return rc;

  const int P = p.P;
  const int n = 6 * P;
  const int64_t S = std::min<int64_t>(p.K, (int64_t)P + p.E);
  const BaLaunch l = ba_launch_shape(p);
  const int nchunk = l.nchunk;
  char* wsb = static_cast<char*>(workspace);
  CholBuf cb{(double*)(wsb + L.L11), (double*)(wsb + L.dinv), (double*)(wsb + L.ychol), (unsigned*)(wsb + L.ctl)};

  for (int it = 0; it < iterations; ++it) {
    if ((rc = build_system(p, l, poses, disps, intrinsics, targets, weights, eta, eta_rows, ii, jj, w, info, s)))
      return rc;
    if ((rc = run_cholesky(n, lm, ep, w, cb, dx, info, s))) return rc;
    if (!p.motion_only && S > 0) {
      dim3 grid((unsigned)S, nchunk);
      HS2_PROF("ba_backsub", s);
      if (g_schur_path.load() == 2) {
        ba_backsub_frame_kernel<<<grid, kLinThreads, 0, s>>>(disps, p.HW, p.wd, intrinsics, weights, jj, t0, t1, w,
                                                             dx, dz, dz_rows, info);
        HS2_LAUNCH_CHECK("ba_backsub_frame_kernel");
      } else {
        ba_backsub_kernel<<<grid, kBsThreads, 0, s>>>(disps, p.HW, P, w, dx, dz, dz_rows, info);
        HS2_LAUNCH_CHECK("ba_backsub_kernel");
      }
    }
    if (P > 0) {
      HS2_PROF("ba_pose_retr", s);
      ba_pose_retr_kernel<<<(P + 127) / 128, 128, 0, s>>>(poses, t0, P, w, info);
      HS2_LAUNCH_CHECK("ba_pose_retr_kernel");
    }
  }
  return HS2_OK;
}

extern "C" int hs2_ba_reduced_system(const float* poses, int64_t num_poses, const float* disps, int64_t num_disps,
                                     int ht, int wd, const float* intrinsics, const float* targets,
                                     const float* weights, const float* eta, int64_t eta_rows, const int64_t* ii,
                                     const int64_t* jj, int64_t num_edges, int t0, int t1, int motion_only,
                                     double* A_out, double* b_out, int32_t* info, void* workspace,
                                     size_t workspace_bytes, hs2_stream_t stream) {
  using namespace hs2;
  BaProblem p = make_problem(num_poses, num_disps, ht, wd, num_edges, t0, t1, motion_only);
  int rc = ba_check(p, "ba_reduced_system");
  if (rc) return rc;
  const BaLayout L = ba_layout(p.K, p.HW, p.E, p.P, p.motion_only);
  if (!workspace || workspace_bytes < L.total) {
    set_error("ba_reduced_system: workspace of %zu bytes required", L.total);
    return HS2_ERR_WORKSPACE;
  }
  if ((rc = bind_device(poses))) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  BaPtrs w = ba_ptrs(workspace, L);
  if ((rc = run_keys(p, ii, jj, motion_only ? 1 : eta_rows, w, info, s))) return rc;
  if ((rc = build_system(p, ba_launch_shape(p), poses, disps, intrinsics, targets, weights, eta, eta_rows, ii, jj,
                         w, info, s)))
    return rc;
  const size_t n = 6 * (size_t)p.P;
  if (n > 0) {
    ba_symmetrize_kernel<<<(unsigned)((n * n + 255) / 256), 256, 0, s>>>((int)n, w.A);
    HS2_LAUNCH_CHECK("ba_symmetrize_kernel");
    HS2_CUDA(cudaMemcpyAsync(A_out, w.A, sizeof(double) * n * n, cudaMemcpyDeviceToDevice, s));
    HS2_CUDA(cudaMemcpyAsync(b_out, w.b, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  }
  return HS2_OK;
}

extern "C" int hs2_ba_set_gram_precision(int precision) {
  using namespace hs2;
  if (precision != 0 && precision != 1) {
    set_error("ba_set_gram_precision: 1 (3xTF32, FP32-accurate) or 0 (one TF32 product)");
    return HS2_ERR_INVALID;
  }
  g_gram_split3.store(precision);
  return HS2_OK;
}

extern "C" int hs2_ba_set_schur_path(int path) {
  using namespace hs2;
  if (path < 0 || path > 2) {
    set_error("ba_set_schur_path: path must be 0 (tensor cores over stored E rows), 1 (SIMT FP32) or 2 (fused, "
              "tensor cores)");
    return HS2_ERR_INVALID;
  }
  g_schur_path.store(path);
  return HS2_OK;
}

namespace hs2 {

// ============================================================ LM adjoint ===
// Adjoint of ONE Levenberg-Marquardt step of ba (motion_only = 0) with respect to
// targets, weights and eta at a fixed linearisation point (poses, disparities):
// implicit differentiation through the damped Schur solve.  With the step written
// as the damped system M_d [dx; dz] = [b; gd] (pose block A + ep + lm diag(R),
// R = A - E Q E^T, depth block C + eta, Q = 1/(C + eta)) and the reference's
// back-substitution dz = Q (gd - E~^T dx) (E~ without the rows of window pose 0,
// EvT6x1_kernel's ix <= 0 skip), the adjoint of (gdx, gdz) is
//   lam   = R_d^-1 (gdx - E~ Q gdz)                          (the forward's Cholesky)
//   per depth pixel k, with s_lam = E_k . lam, s_x = E_k . dx, s~_x = E~_k . dx and
//   e2 = sum over pose dofs of lam dx E_k^2 (E_k summed over rows of one pose):
//     Qbar  = gdz (gd - s~_x) - s_lam gd + s_lam s_x + lm e2
//     gdbar = Q (gdz - s_lam),   Cbar = etabar = -Q^2 Qbar
//   per edge-pixel and channel, with u = J . lam, v = J . dx, v~ (without pose 0),
//   J_d the depth Jacobian, r the residual and w' = 0.001 weight (0 when z < MIN_DEPTH):
//     wbar' = -u v - lm sum lam dx J^2 + u r
//             + J_d Q (-gdz v~ - gd u + s_x u + s_lam v + 2 lm sum J lam dx E)   (pose terms)
//             + Cbar J_d^2 + gdbar J_d r                                          (depth terms)
//     weights_bar = 0.001 valid wbar',  targets_bar = w' u + gdbar w' J_d
// (self-edges keep only the depth terms, as in the forward).  R_bar = -lam dx^T -
// lm diag(lam dx) is rank two plus a diagonal, which is why every term above needs
// only the per-pixel scalars and no second Gram.
constexpr int kAdjThreads = 128;
constexpr int kAdjMaxRows = 256;     // Schur rows of one depth frame held in shared memory

// rhs[a*6+x] = sum over Schur rows of pose a >= 1 of sum_p E Q gdz (FP64 accumulation)
__global__ void __launch_bounds__(kAdjThreads)
ba_adj_rhs_kernel(int HW, BaPtrs w, const float* __restrict__ gdz, double* __restrict__ acc,
                  const int32_t* __restrict__ info) {
  if (info[0]) return;
  const int s = blockIdx.x;
  if (s >= info[1]) return;
  const int HWs = row_stride(HW);
  const int q0 = w.sptr[s], q1 = w.sptr[s + 1];
  __shared__ float red[kAdjThreads / 32][6];
  for (int q = q0; q < q1; ++q) {
    const int pose = w.spose[q];
    if (pose < 1) continue;
    const int r = w.rptr[s] + (q - q0);
    float part[6] = {0, 0, 0, 0, 0, 0};
    for (int p = blockIdx.y * blockDim.x + threadIdx.x; p < HW; p += gridDim.y * blockDim.x) {
      const float qz = w.qbuf[(int64_t)s * HW + p] * gdz[(int64_t)s * HW + p];
#pragma unroll
      for (int x = 0; x < 6; ++x) part[x] = fmaf(w.erows[((int64_t)r * 6 + x) * HWs + p], qz, part[x]);
    }
#pragma unroll
    for (int x = 0; x < 6; ++x) part[x] = warp_sum(part[x]);
    __syncthreads();
    if ((threadIdx.x & 31) == 0)
      for (int x = 0; x < 6; ++x) red[threadIdx.x >> 5][x] = part[x];
    __syncthreads();
    if (threadIdx.x < 6) {
      double t = 0.0;
      for (int k = 0; k < kAdjThreads / 32; ++k) t += red[k][threadIdx.x];
      atomicAdd(&acc[pose * 6 + threadIdx.x], t);
    }
  }
}

__global__ void ba_adj_b_kernel(int n, const float* __restrict__ gdx, const double* __restrict__ acc,
                                double* __restrict__ b, const int32_t* __restrict__ info) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || info[0]) return;
  b[i] = (double)gdx[i] - acc[i];
}

// Per depth pixel: s_lam, s_x, gdbar, Cbar (stored for the edge kernel) and etabar.
__global__ void __launch_bounds__(kAdjThreads)
ba_adj_pixel_kernel(int HW, BaPtrs w, const float* __restrict__ lam, const float* __restrict__ dx,
                    const float* __restrict__ gdz, float lm, int64_t eta_rows, float* __restrict__ pix,
                    float* __restrict__ geta, const int32_t* __restrict__ info) {
  if (info[0]) return;
  const int s = blockIdx.x;
  const int M = info[1];
  if (s >= M) return;
  const int HWs = row_stride(HW);
  const int q0 = w.sptr[s], nq = min(w.sptr[s + 1] - q0, kAdjMaxRows);
  if (w.sptr[s + 1] - q0 > kAdjMaxRows) {
    if (threadIdx.x == 0 && blockIdx.y == 0) atomicOr((int32_t*)info, HS2_DEV_LIMIT);
    return;
  }
  __shared__ int pose[kAdjMaxRows], first[kAdjMaxRows], nxt[kAdjMaxRows];
  for (int q = threadIdx.x; q < nq; q += blockDim.x) pose[q] = w.spose[q0 + q];
  __syncthreads();
  for (int q = threadIdx.x; q < nq; q += blockDim.x) {
    int f = 1, n = -1;
    for (int k = 0; k < q; ++k) f &= pose[k] != pose[q];
    for (int k = nq - 1; k > q; --k)
      if (pose[k] == pose[q]) n = k;
    first[q] = f;
    nxt[q] = n;
  }
  __syncthreads();
  const int rbase = w.rptr[s];
  const int p = blockIdx.y * blockDim.x + threadIdx.x;
  if (p >= HW) return;
  float sl = 0.f, sx = 0.f, sxt = 0.f, e2 = 0.f;
  for (int q = 0; q < nq; ++q) {
    if (!first[q]) continue;
    const int a = pose[q];
    float e[6];
#pragma unroll
    for (int x = 0; x < 6; ++x) e[x] = 0.f;
    for (int k = q; k >= 0; k = nxt[k]) {
#pragma unroll
      for (int x = 0; x < 6; ++x) e[x] += w.erows[((int64_t)(rbase + k) * 6 + x) * HWs + p];
    }
#pragma unroll
    for (int x = 0; x < 6; ++x) {
      const float l = lam[a * 6 + x], d = dx[a * 6 + x];
      sl = fmaf(e[x], l, sl);
      sx = fmaf(e[x], d, sx);
      if (a >= 1) sxt = fmaf(e[x], d, sxt);
      e2 = fmaf(l * d, e[x] * e[x], e2);
    }
  }
  const int64_t k = (int64_t)s * HW + p;
  const float Q = w.qbuf[k], gd = w.wbuf[k], zb = gdz[k];
  const float Qbar = zb * (gd - sxt) - sl * gd + sl * sx + lm * e2;
  const float gdbar = Q * (zb - sl);
  const float Cbar = -Q * Q * Qbar;
  const int64_t MHW = (int64_t)M * HW;
  pix[k] = sl;
  pix[MHW + k] = sx;
  pix[2 * MHW + k] = gdbar;
  pix[3 * MHW + k] = Cbar;
  if (eta_rows == 1) atomicAdd(&geta[p], Cbar);
  else geta[k] = Cbar;
}

// Per edge-pixel: the linearisation again (lin_pixel's arithmetic), then the
// gradients of the edge's targets and weights.
__global__ void __launch_bounds__(kAdjThreads)
ba_adj_edge_kernel(const float* __restrict__ disps, int HW, int wd, const float* __restrict__ intr,
                   const float* __restrict__ targets, const float* __restrict__ weights,
                   const int64_t* __restrict__ ii, const int64_t* __restrict__ jj, int t0, int P, BaPtrs w,
                   const float* __restrict__ lam, const float* __restrict__ dx, const float* __restrict__ gdz,
                   float lm, const float* __restrict__ pix, float* __restrict__ gt, float* __restrict__ gw,
                   const int32_t* __restrict__ info) {
  if (info[0]) return;
  const int e = blockIdx.x;
  const int M = info[1];
  const int HWs = row_stride(HW);
  __shared__ float tab[kEtab];
  __shared__ float sl_a[6], sd_a[6], sl_b[6], sd_b[6];
  __shared__ int rows_a[8], rows_b[8], nra, nrb;
  const int f = (int)ii[e], g = (int)jj[e];
  const int s = w.slot[f];
  const int a = f - t0, b = g - t0;
  const bool ina = a >= 0 && a < P, inb = b >= 0 && b < P, self = f == g;
  if (threadIdx.x < kEtab) tab[threadIdx.x] = w.etab[(int64_t)e * kEtab + threadIdx.x];
  if (threadIdx.x < 6) {
    sl_a[threadIdx.x] = ina ? lam[a * 6 + threadIdx.x] : 0.f;
    sd_a[threadIdx.x] = ina ? dx[a * 6 + threadIdx.x] : 0.f;
    sl_b[threadIdx.x] = inb ? lam[b * 6 + threadIdx.x] : 0.f;
    sd_b[threadIdx.x] = inb ? dx[b * 6 + threadIdx.x] : 0.f;
  }
  if (threadIdx.x == 0) {
    // storage rows of pose a and pose b among the Schur rows of the edge's depth frame
    int na = 0, nb = 0;
    const int q0 = w.sptr[s], q1 = w.sptr[s + 1];
    for (int q = q0; q < q1; ++q) {
      const int pz = w.spose[q];
      if (pz == a) {
        if (na < 8) rows_a[na] = w.rptr[s] + (q - q0);
        ++na;
      }
      if (pz == b) {
        if (nb < 8) rows_b[nb] = w.rptr[s] + (q - q0);
        ++nb;
      }
    }
    if ((na > 8 || nb > 8) && blockIdx.y == 0) atomicOr((int32_t*)info, HS2_DEV_LIMIT);
    na = min(na, 8);
    nb = min(nb, 8);
    nra = na;
    nrb = nb;
  }
  __syncthreads();
  const int p = blockIdx.y * blockDim.x + threadIdx.x;
  if (p >= HW) return;
  const float fx = intr[0], fy = intr[1], cx = intr[2], cy = intr[3];
  const int vi = p / wd;
  const float xn = ((float)(p - vi * wd) - cx) / fx, yn = ((float)vi - cy) / fy;
  const float h = disps[(int64_t)f * HW + p];
  const float* R = tab + 44;
  const float Y0 = fmaf(R[0], xn, fmaf(R[1], yn, R[2])) + h * tab[0];
  const float Y1 = fmaf(R[3], xn, fmaf(R[4], yn, R[5])) + h * tab[1];
  const float Y2 = fmaf(R[6], xn, fmaf(R[7], yn, R[8])) + h * tab[2];
  const bool bad = Y2 < kMinDepth;
  const float iz = __fdividef(1.0f, Y2);
  const float proj[2] = {fx * (Y0 * iz) + cx, fy * (Y1 * iz) + cy};
  const float z = bad ? 0.f : Y2, dd = bad ? 0.f : iz, d2 = dd * dd;
  const float Jp0 = fx * dd, Jp2 = fx * (-Y0 * d2), Jp4 = fy * dd, Jp5 = fy * (-Y1 * d2);
  const float Jc[2][6] = {{Jp0 * h, 0.f, Jp2 * h, Jp2 * Y1, Jp0 * z - Jp2 * Y0, -Jp0 * Y1},
                          {0.f, Jp4 * h, Jp5 * h, -Jp4 * z + Jp5 * Y1, -Jp5 * Y0, Jp4 * Y0}};
  const float Jd[2] = {Jp0 * tab[0] + Jp2 * tab[2], Jp4 * tab[1] + Jp5 * tab[2]};
  float Ea[6], Eb[6];
#pragma unroll
  for (int x = 0; x < 6; ++x) { Ea[x] = 0.f; Eb[x] = 0.f; }
  for (int k = 0; k < nra; ++k)
#pragma unroll
    for (int x = 0; x < 6; ++x) Ea[x] += w.erows[((int64_t)rows_a[k] * 6 + x) * HWs + p];
  for (int k = 0; k < nrb; ++k)
#pragma unroll
    for (int x = 0; x < 6; ++x) Eb[x] += w.erows[((int64_t)rows_b[k] * 6 + x) * HWs + p];
  const int64_t kp = (int64_t)s * HW + p;
  const int64_t MHW = (int64_t)M * HW;
  const float sl = pix[kp], sx = pix[MHW + kp], gdbar = pix[2 * MHW + kp], Cbar = pix[3 * MHW + kp];
  const float Q = w.qbuf[kp], gd = w.wbuf[kp], zb = gdz[kp];
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    const int64_t o = ((int64_t)e * 2 + c) * HW + p;
    const float wgt = bad ? 0.f : 0.001f * weights[o];
    const float r = targets[o] - proj[c];
    // Ji = L Jj (L from the edge table, as the forward's Ei = L Ej)
    float Ji[6];
#pragma unroll
    for (int x = 0; x < 6; ++x) {
      float t = 0.f;
#pragma unroll
      for (int y = 0; y < 6; ++y) t = fmaf(tab[8 + x * 6 + y], Jc[c][y], t);
      Ji[x] = t;
    }
    float u = 0.f, v = 0.f, vt = 0.f, dmp = 0.f, eb = 0.f;
#pragma unroll
    for (int x = 0; x < 6; ++x) {
      const float ja = ina ? Ji[x] : 0.f, jb = inb ? Jc[c][x] : 0.f;
      u += ja * sl_a[x] + jb * sl_b[x];
      v += ja * sd_a[x] + jb * sd_b[x];
      vt += (a >= 1 ? ja * sd_a[x] : 0.f) + (b >= 1 ? jb * sd_b[x] : 0.f);
      dmp += ja * ja * sl_a[x] * sd_a[x] + jb * jb * sl_b[x] * sd_b[x];
      eb += ja * sl_a[x] * sd_a[x] * Ea[x] + jb * sl_b[x] * sd_b[x] * Eb[x];
    }
    float wb = Cbar * Jd[c] * Jd[c] + gdbar * Jd[c] * r;
    float tb = gdbar * wgt * Jd[c];
    if (!self) {
      wb += -u * v - lm * dmp + u * r + Jd[c] * Q * (-zb * vt - gd * u + sx * u + sl * v + 2.f * lm * eb);
      tb += wgt * u;
    }
    gw[o] = bad ? 0.f : 0.001f * wb;
    gt[o] = tb;
  }
}

static size_t ba_adj_extra(int64_t M, int HW, int P) {
  return align256(sizeof(double) * (6 * (size_t)P + 1)) + align256(sizeof(float) * (6 * (size_t)P + 1)) +
         align256(sizeof(float) * 4 * (size_t)M * HW);
}

}  // namespace hs2

extern "C" int hs2_ba_adjoint_workspace_size(int64_t num_poses, int64_t num_disps, int ht, int wd,
                                             int64_t num_edges, int t0, int t1, size_t* bytes) {
  using namespace hs2;
  if (!bytes) {
    set_error("ba_adjoint_workspace_size: null output");
    return HS2_ERR_INVALID;
  }
  BaProblem p = make_problem(num_poses, num_disps, ht, wd, num_edges, t0, t1, 0);
  int rc = ba_check(p, "ba_adjoint_workspace_size");
  if (rc) return rc;
  const int64_t S = std::min<int64_t>(p.K, (int64_t)p.P + p.E);
  *bytes = ba_layout(p.K, p.HW, p.E, p.P, 0).total + ba_adj_extra(S, p.HW, p.P);
  return HS2_OK;
}

extern "C" int hs2_ba_adjoint(const float* poses, int64_t num_poses, const float* disps, int64_t num_disps, int ht,
                              int wd, const float* intrinsics, const float* targets, const float* weights,
                              const float* eta, int64_t eta_rows, const int64_t* ii, const int64_t* jj,
                              int64_t num_edges, int t0, int t1, float lm, float ep, const float* dx,
                              const float* grad_dx, const float* grad_dz, int64_t dz_rows, float* grad_targets,
                              float* grad_weights, float* grad_eta, float* lam, int32_t* info, void* workspace,
                              size_t workspace_bytes, hs2_stream_t stream) {
  using namespace hs2;
  BaProblem p = make_problem(num_poses, num_disps, ht, wd, num_edges, t0, t1, 0);
  int rc = ba_check(p, "ba_adjoint");
  if (rc) return rc;
  const BaLayout L = ba_layout(p.K, p.HW, p.E, p.P, 0);
  const int64_t S = std::min<int64_t>(p.K, (int64_t)p.P + p.E);
  const size_t need = L.total + ba_adj_extra(S, p.HW, p.P);
  if (!workspace || workspace_bytes < need) {
    set_error("ba_adjoint: workspace of %zu bytes required", need);
    return HS2_ERR_WORKSPACE;
  }
  if (!lam || !info || (p.E > 0 && (!grad_targets || !grad_weights)) || !grad_eta || (p.P > 0 && (!dx || !grad_dx))) {
    set_error("ba_adjoint: null output or input pointer");
    return HS2_ERR_INVALID;
  }
  if ((rc = bind_device(poses))) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  BaPtrs w = ba_ptrs(workspace, L);
  char* extra = static_cast<char*>(workspace) + L.total;
  double* acc = reinterpret_cast<double*>(extra);
  float* pix = reinterpret_cast<float*>(extra + align256(sizeof(double) * (6 * (size_t)p.P + 1)) +
                                        align256(sizeof(float) * (6 * (size_t)p.P + 1)));
  if ((rc = run_keys(p, ii, jj, eta_rows, w, info, s))) return rc;
  const int P = p.P;
  const int n = 6 * P;
  HS2_CUDA(cudaMemsetAsync(grad_eta, 0, sizeof(float) * (size_t)eta_rows * p.HW, s));
  if (p.E > 0) {
    HS2_CUDA(cudaMemsetAsync(grad_targets, 0, sizeof(float) * 2 * (size_t)p.E * p.HW, s));
    HS2_CUDA(cudaMemsetAsync(grad_weights, 0, sizeof(float) * 2 * (size_t)p.E * p.HW, s));
  }
  if (S == 0) return HS2_OK;
  const BaLaunch l = ba_launch_shape(p);
  if ((rc = build_system(p, l, poses, disps, intrinsics, targets, weights, eta, eta_rows, ii, jj, w, info, s)))
    return rc;
  const int chunks = (p.HW + kAdjThreads - 1) / kAdjThreads;
  if (n > 0) {
    HS2_CUDA(cudaMemsetAsync(acc, 0, sizeof(double) * n, s));
    HS2_PROF("ba_adj_rhs", s);
    ba_adj_rhs_kernel<<<dim3((unsigned)S, std::min(chunks, 8)), kAdjThreads, 0, s>>>(p.HW, w, grad_dz, acc, info);
    HS2_LAUNCH_CHECK("ba_adj_rhs_kernel");
    ba_adj_b_kernel<<<(n + 255) / 256, 256, 0, s>>>(n, grad_dx, acc, w.b, info);
    HS2_LAUNCH_CHECK("ba_adj_b_kernel");
    char* wsb = static_cast<char*>(workspace);
    CholBuf cb{(double*)(wsb + L.L11), (double*)(wsb + L.dinv), (double*)(wsb + L.ychol), (unsigned*)(wsb + L.ctl)};
    if ((rc = run_cholesky(n, lm, ep, w, cb, lam, info, s))) return rc;
  }
  {
    HS2_PROF("ba_adj_pixel", s);
    ba_adj_pixel_kernel<<<dim3((unsigned)S, chunks), kAdjThreads, 0, s>>>(p.HW, w, lam, dx, grad_dz, lm, eta_rows,
                                                                         pix, grad_eta, info);
    HS2_LAUNCH_CHECK("ba_adj_pixel_kernel");
  }
  if (p.E > 0) {
    HS2_PROF("ba_adj_edge", s);
    ba_adj_edge_kernel<<<dim3((unsigned)p.E, chunks), kAdjThreads, 0, s>>>(
        disps, p.HW, p.wd, intrinsics, targets, weights, ii, jj, t0, P, w, lam, dx, grad_dz, lm, pix, grad_targets,
        grad_weights, info);
    HS2_LAUNCH_CHECK("ba_adj_edge_kernel");
  }
  return HS2_OK;
}

namespace hs2 {

}  // namespace hs2

// ================================================================= pgba ===
// Sim3 pose-graph bundle adjustment (reference operator: src/droid.cpp:171-196 ->
// src/droid_kernels.cu:1940-2044): ONE damped Gauss-Newton step over Sim3 poses
// [t(3), q(4), s] (7-dof tangent [tau, phi, sigma]) and per-pixel inverse depths, with
// the caller's relative-pose factors added to the pose system.  Poses are not moved
// (dx is returned for the caller's Sim3 retraction); disparities are updated in place.
//
//   keys        as for ba (ba_keys_kernel): depth frames kx, edge groups, row lists
//   pg_edge     Gij = Gj Gi^-1 (Sim3) and the 7x7 map L with Ji = L Jj, L = -adjSim3
//               as the reference writes it (:122-145; its rotation and scale columns
//               are not the derivative of the reprojection, and are kept for parity)
//   pg_linearize per (depth frame, pixel chunk): residuals and Sim3 Jacobians of every
//               edge leaving the frame (:608-858): each edge's Hjj / vj summed in FP64,
//               its E row written, the frame's Ei = sum L Eij row, Q = 1/(C + eta), w
//   pg_assemble Hii = L Hjj L^T, Hij = L Hjj, vi = L vj into the FP64 system (keys - t0,
//               negatives dropped: SparseBlock::update_lhs/update_rhs :1598-1638)
//   pg_prior    the relative-pose blocks Hsp / vsp at iip, jjp (:2004-2013)
//   pg_schur    per depth frame the Gram of its Schur rows weighted by Q, subtracted
//               (schur_block + EEt6x6 + Ev6x1 at D = 7, :1466-1560, :1689-1779)
//   cholesky    the BA kernel on the system padded to even order with an identity row
//   pg_backsub  dz = Q (w - sum E.dx) with the reference's ix <= 0 skip, disps += dz
// Only the lower triangle (with whole diagonal blocks) of the reduced matrix is
// written and read, as the reference's SimplicialLLT reads it: a block at keys (R, C)
// is added when R >= C.
namespace hs2 {

constexpr int kPgD = 7;
constexpr int kPgTab = 72;        // floats per edge: t 0..2, q 3..6, s 7, L 8..56 (row-major), s R 57..65
constexpr int kPgH = 35;          // upper triangle of Hjj (28), then vj (7)
// pg_linearize: 128 threads x 4 pixels (four CTAs per SM); pg_backsub: 256 threads x 2
// pixels over the same 512-pixel chunks (measured: 0.63 / 0.16 ms at 300 kf against
// 0.67 / 0.20 ms with 256 x 4 for both)
constexpr int kPgThreads = 128;
constexpr int kPgPPT = 4;
constexpr int kPgChunk = kPgThreads * kPgPPT;
constexpr int kPgBsThreads = 256;
constexpr int kPgBsPPT = 2;
static_assert(kPgBsThreads * kPgBsPPT == kPgChunk, "pg_backsub covers the linearisation's chunks");
constexpr int kPgSplit = 16;      // CTAs per depth frame in the Gram

__host__ __device__ __forceinline__ int64_t pg_order(int P) { return 7 * (int64_t)P + ((7 * (int64_t)P) & 1); }

__device__ __forceinline__ int tri7(int r, int c) { return r * 7 - (r * (r - 1)) / 2 + (c - r); }

__global__ void pg_edge_kernel(const float* __restrict__ poses, const int64_t* __restrict__ ii,
                               const int64_t* __restrict__ jj, int E, float* __restrict__ ptab,
                               double* __restrict__ L64, const int32_t* __restrict__ info) {
  const int gid = blockIdx.x * blockDim.x + threadIdx.x;
  const int e = gid / 7, c = gid - (gid / 7) * 7;
  if (e >= E || info[0]) return;
  const float* pi = poses + 8 * ii[e];
  const float* pj = poses + 8 * jj[e];
  const double ti[3] = {pi[0], pi[1], pi[2]}, qi[4] = {pi[3], pi[4], pi[5], pi[6]};
  const double tj[3] = {pj[0], pj[1], pj[2]}, qj[4] = {pj[3], pj[4], pj[5], pj[6]};
  double t_se3[3], q[4], rti[3];
  relative_pose(ti, qi, tj, qj, t_se3, q);   // qij = qj conj(qi)
  quat_rotate(q, ti, rti);
  const double sij = (double)pj[7] / (double)pi[7];
  const double t[3] = {tj[0] - sij * rti[0], tj[1] - sij * rti[1], tj[2] - sij * rti[2]};
  float* tab = ptab + (int64_t)e * kPgTab;
  if (c == 0) {
    for (int k = 0; k < 3; ++k) tab[k] = (float)t[k];
    for (int k = 0; k < 4; ++k) tab[3 + k] = (float)q[k];
    tab[7] = (float)sij;
    const double x = q[0], y = q[1], z = q[2], w = q[3];
    const double R[9] = {1 - 2 * (y * y + z * z), 2 * (x * y - z * w),     2 * (x * z + y * w),
                         2 * (x * y + z * w),     1 - 2 * (x * x + z * z), 2 * (y * z - x * w),
                         2 * (x * z - y * w),     2 * (y * z + x * w),     1 - 2 * (x * x + y * y)};
    for (int k = 0; k < 9; ++k) tab[57 + k] = (float)(sij * R[k]);
    for (int k = 66; k < kPgTab; ++k) tab[k] = 0.f;
  }
  // column c of L: Ji for Jj = unit vector c.  -adjSim3 (:122-145):
  //   Ji[0:3] = s (-R^T a),  Ji[3:6] = s (-R^T (b + a x t)) - c6 t,  Ji[6] = -c6
  double u[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) u[k] = k == c ? 1.0 : 0.0;
  const double c6 = c == 6 ? 1.0 : 0.0;
  double r[6];
  pose_jacobian_i(t, q, u, r);
  double col[7];
  for (int k = 0; k < 3; ++k) col[k] = sij * r[k];
  for (int k = 0; k < 3; ++k) col[3 + k] = sij * r[3 + k] - c6 * t[k];
  col[6] = -c6;
  for (int k = 0; k < 7; ++k) {
    tab[8 + k * 7 + c] = (float)col[k];
    L64[(int64_t)e * 49 + k * 7 + c] = col[k];
  }
}

// One CTA per (depth frame slot, chunk of kPgChunk pixels); thread t owns the pixels
// t + kPgThreads k.  For every edge of the frame (in group order) each pixel is moved by
// Gij, projected and linearised as the reference does per pixel (:700-814); the
// edge's 35 Hessian sums are reduced over the CTA into FP64 accumulators.
__global__ void __launch_bounds__(kPgThreads, 4)
pg_linearize_kernel(const float* __restrict__ disps, int HW, int wd, const float* __restrict__ intr,
                    const float* __restrict__ targets, const float* __restrict__ weights,
                    const float* __restrict__ eta, int64_t eta_rows, const int64_t* __restrict__ jj, int t0,
                    int t1, const float* __restrict__ ptab, BaPtrs w, float* __restrict__ erows,
                    float* __restrict__ qbuf, float* __restrict__ wbuf, double* __restrict__ hedge,
                    const int32_t* __restrict__ info) {
  if (info[0]) return;
  const int s = blockIdx.x;
  if (s >= info[1]) return;
  const int f = w.kx[s];
  const bool inwin = f >= t0 && f < t1;
  const size_t HWs = (size_t)row_stride(HW);
  __shared__ float tab[kPgTab];
  __shared__ float red[kPgThreads / 32][kPgH];
  const float fx = intr[0], fy = intr[1], cx = intr[2], cy = intr[3];
  const int base = blockIdx.y * kPgChunk + threadIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  float xn[kPgPPT], yn[kPgPPT], hd[kPgPPT], C[kPgPPT], W[kPgPPT], Ei[kPgPPT][kPgD];
#pragma unroll
  for (int k = 0; k < kPgPPT; ++k) {
    const int p = base + k * kPgThreads;
    const bool ok = p < HW;
    xn[k] = ok ? ((float)(p % wd) - cx) / fx : 0.f;
    yn[k] = ok ? ((float)(p / wd) - cy) / fy : 0.f;
    hd[k] = ok ? disps[(int64_t)f * HW + p] : 0.f;
    C[k] = 0.f;
    W[k] = 0.f;
#pragma unroll
    for (int d = 0; d < kPgD; ++d) Ei[k][d] = 0.f;
  }
  for (int g = w.gptr[s]; g < w.gptr[s + 1]; ++g) {
    const int e = w.gedge[g];
    __syncthreads();   // tab / red of the previous edge are consumed
    if (threadIdx.x < kPgTab) tab[threadIdx.x] = ptab[(int64_t)e * kPgTab + threadIdx.x];
    __syncthreads();
    const bool self = jj[e] == (int64_t)f;
    const size_t row = (size_t)w.epos[e];
    const float* tg = targets + (int64_t)e * 2 * HW;
    const float* wg = weights + (int64_t)e * 2 * HW;
    float h[kPgH];
#pragma unroll
    for (int i = 0; i < kPgH; ++i) h[i] = 0.f;
#pragma unroll
    for (int k = 0; k < kPgPPT; ++k) {
      const int p = base + k * kPgThreads;
      if (p >= HW) continue;
      // Xj = s R X + h t with X = (xn, yn, 1) (actSim3 :96-102)
      const float x = tab[57] * xn[k] + tab[58] * yn[k] + tab[59] + hd[k] * tab[0];
      const float y = tab[60] * xn[k] + tab[61] * yn[k] + tab[62] + hd[k] * tab[1];
      const float Z = tab[63] * xn[k] + tab[64] * yn[k] + tab[65] + hd[k] * tab[2];
      const float hh = hd[k];
      const bool bad = Z < kMinDepth;
      const float z = bad ? 0.f : Z;
      const float dd = bad ? 0.f : 1.f / Z;
      const float d2 = dd * dd;
      float wu = bad ? 0.f : 0.001f * wg[p];
      float wv = bad ? 0.f : 0.001f * wg[HW + p];
      const float ru = tg[p] - (fx * (x / Z) + cx);
      const float rv = tg[HW + p] - (fy * (y / Z) + cy);
      const float Jp0 = fx * dd, Jp2 = fx * (-x * d2), Jp4 = fy * dd, Jp5 = fy * (-y * d2);
      const float Jzu = Jp0 * tab[0] + Jp2 * tab[2];
      const float Jzv = Jp4 * tab[1] + Jp5 * tab[2];
      C[k] += wu * Jzu * Jzu + wv * Jzv * Jzv;
      W[k] += wu * ru * Jzu + wv * rv * Jzv;
      if (self) {
        wu = 0.f;
        wv = 0.f;
      }
      // Jj rows of u and v (:733-740, :767-774; Jp[1] = Jp[3] = 0)
      const float Ju[kPgD] = {Jp0 * hh, 0.f, Jp2 * hh, Jp2 * y, Jp0 * z - Jp2 * x, -Jp0 * y, Jp0 * x + Jp2 * z};
      const float Jv[kPgD] = {0.f, Jp4 * hh, Jp5 * hh, -Jp4 * z + Jp5 * y, -Jp5 * x, Jp4 * x, Jp4 * y + Jp5 * z};
#pragma unroll
      for (int a = 0; a < kPgD; ++a) {
#pragma unroll
        for (int b = a; b < kPgD; ++b) h[tri7(a, b)] += wu * Ju[a] * Ju[b] + wv * Jv[a] * Jv[b];
        h[28 + a] += wu * ru * Ju[a] + wv * rv * Jv[a];
      }
      float ej[kPgD];
#pragma unroll
      for (int a = 0; a < kPgD; ++a) {
        ej[a] = wu * Jzu * Ju[a] + wv * Jzv * Jv[a];
        erows[(row * kPgD + a) * HWs + p] = ej[a];
      }
      if (inwin) {
#pragma unroll
        for (int r = 0; r < kPgD; ++r) {
          float acc = 0.f;
#pragma unroll
          for (int c = 0; c < kPgD; ++c) acc += tab[8 + r * 7 + c] * ej[c];
          Ei[k][r] += acc;
        }
      }
    }
    {
      // the first 32 sums by the transpose exchange (lane l ends with the total of h[l]),
      // the remaining ones by plain butterflies
      static_assert(kPgH >= 32, "pg_linearize: at least 32 sums per edge");
#pragma unroll
      for (int i = 32; i < kPgH; ++i) {
        const float v = warp_sum(h[i]);
        if (lane == 0) red[warp][i] = v;
      }
      red[warp][lane] = warp_transpose_sum(*reinterpret_cast<float(*)[32]>(h));   // consumes h[0..31]
    }
    __syncthreads();
    if (threadIdx.x < kPgH) {
      double acc = 0.0;
#pragma unroll
      for (int q = 0; q < kPgThreads / 32; ++q) acc += (double)red[q][threadIdx.x];
      atomicAdd(&hedge[(int64_t)e * kPgH + threadIdx.x], acc);
    }
  }
  const int64_t er = eta_rows == 1 ? 0 : s;
  const size_t wrow = inwin ? (size_t)w.wpos[f - t0] : 0;
#pragma unroll
  for (int k = 0; k < kPgPPT; ++k) {
    const int p = base + k * kPgThreads;
    if (p >= HW) continue;
    qbuf[(int64_t)s * HW + p] = 1.f / (C[k] + eta[er * HW + p]);
    wbuf[(int64_t)s * HW + p] = W[k];
    if (inwin) {
#pragma unroll
      for (int d = 0; d < kPgD; ++d) erows[(wrow * kPgD + d) * HWs + p] = Ei[k][d];
    }
  }
}

// Adds row r of a 7x7 block to the system at block keys (R, C) when R >= C (lower
// triangle with whole diagonal blocks); negative keys are dropped.
__device__ __forceinline__ void pg_add_row(double* A, int64_t npad, int R, int C, int r, const double* v) {
  if (R < 0 || C < 0 || R < C) return;
  double* dst = A + (7 * (int64_t)R + r) * npad + 7 * (int64_t)C;
#pragma unroll
  for (int c = 0; c < kPgD; ++c) atomicAdd(dst + c, v[c]);
}

// Seven threads per edge, thread r forms row r of Hii, Hij, Hji^T's column and Hjj.
__global__ void pg_assemble_kernel(const int64_t* __restrict__ ii, const int64_t* __restrict__ jj, int E, int t0,
                                   int64_t npad, const double* __restrict__ L64, const double* __restrict__ hedge,
                                   double* __restrict__ A, double* __restrict__ b, const int32_t* __restrict__ info) {
  const int gid = blockIdx.x * blockDim.x + threadIdx.x;
  const int e = gid / 7, r = gid - (gid / 7) * 7;
  if (e >= E || info[0]) return;
  const int i = (int)(ii[e] - t0), j = (int)(jj[e] - t0);
  const double* H = hedge + (int64_t)e * kPgH;
  const double* L = L64 + (int64_t)e * 49;
  double hjj_r[kPgD], hij_r[kPgD], hii_r[kPgD];
#pragma unroll
  for (int c = 0; c < kPgD; ++c) hjj_r[c] = H[r <= c ? tri7(r, c) : tri7(c, r)];
  double vi = 0.0;
#pragma unroll
  for (int c = 0; c < kPgD; ++c) {
    double acc = 0.0;
#pragma unroll
    for (int k = 0; k < kPgD; ++k) acc += L[r * 7 + k] * H[k <= c ? tri7(k, c) : tri7(c, k)];
    hij_r[c] = acc;
    vi += L[r * 7 + c] * H[28 + c];
  }
#pragma unroll
  for (int c = 0; c < kPgD; ++c) {
    double acc = 0.0;
#pragma unroll
    for (int k = 0; k < kPgD; ++k) acc += hij_r[k] * L[c * 7 + k];
    hii_r[c] = acc;
  }
  pg_add_row(A, npad, i, i, r, hii_r);
  pg_add_row(A, npad, i, j, r, hij_r);
  pg_add_row(A, npad, j, j, r, hjj_r);
  // Hji = Hij^T: row r of Hij is column r of the block at (j, i)
  if (j >= 0 && i >= 0 && j >= i) {
    double* dst = A + 7 * (int64_t)j * npad + 7 * (int64_t)i + r;
#pragma unroll
    for (int c = 0; c < kPgD; ++c) atomicAdd(dst + c * npad, hij_r[c]);
  }
  if (i >= 0) atomicAdd(&b[7 * (int64_t)i + r], vi);
  if (j >= 0) atomicAdd(&b[7 * (int64_t)j + r], H[28 + r]);
}

// Seven threads per relative-pose factor p: blocks Hsp[0..3][p] at (iip,iip), (iip,jjp),
// (jjp,iip), (jjp,jjp) and vsp[0..1][p] at iip, jjp.  Keys >= t1 are refused.
__global__ void pg_prior_kernel(const float* __restrict__ Hsp, const float* __restrict__ vsp,
                                const int64_t* __restrict__ iip, const int64_t* __restrict__ jjp, int64_t Np,
                                int t0, int t1, int64_t npad, double* __restrict__ A, double* __restrict__ b,
                                int32_t* __restrict__ info) {
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t p = gid / 7;
  const int r = (int)(gid - p * 7);
  if (p >= Np || info[0]) return;
  const int64_t a = iip[p], c = jjp[p];
  if (a >= t1 || c >= t1) {
    atomicOr(info, HS2_DEV_BAD_INDEX);
    return;
  }
  const int i = a < t0 ? -1 : (int)(a - t0), j = c < t0 ? -1 : (int)(c - t0);
  const int keys[4][2] = {{i, i}, {i, j}, {j, i}, {j, j}};
  for (int blk = 0; blk < 4; ++blk) {
    const float* src = Hsp + ((int64_t)blk * Np + p) * 49 + r * 7;
    double v[kPgD];
#pragma unroll
    for (int k = 0; k < kPgD; ++k) v[k] = (double)src[k];
    pg_add_row(A, npad, keys[blk][0], keys[blk][1], r, v);
  }
  if (i >= 0) atomicAdd(&b[7 * (int64_t)i + r], (double)vsp[p * 7 + r]);
  if (j >= 0) atomicAdd(&b[7 * (int64_t)j + r], (double)vsp[(Np + p) * 7 + r]);
}

__global__ void pg_pad_kernel(double* __restrict__ A, int64_t n, int64_t npad) {
  if (threadIdx.x == 0 && blockIdx.x == 0 && npad > n) A[n * npad + n] = 1.0;
}

// Gram of a frame's Schur rows (stored at rptr[s] + a, a < nr, in srow order): 32 x 32 output tiles
// of the (7 R) x (7 R) matrix G_xy = sum_p E_x Q E_y, lower tiles only, spread over
// gridDim.y CTAs of 64 threads.  Pixels are staged 32 at a time k-major in shared memory
// (thread (rh, pc) loads pixel column pc of rows rh, rh + 2, ..); each thread keeps a
// 4 x 4 block of outputs and reads its operands as float4.  Each unordered pair {x, y}
// of the full Gram is subtracted once at the lower-triangle position of the system it
// maps to (twice onto a diagonal entry hit by both orders).
constexpr int kPgGT = 32;   // Gram tile (outputs per side)
constexpr int kPgGK = 32;   // pixels per stage
constexpr int kPgGThreads = 64;

__global__ void __launch_bounds__(kPgGThreads)
pg_schur_kernel(int HW, int64_t npad, BaPtrs w, const float* __restrict__ erows, const float* __restrict__ qbuf,
                double* __restrict__ A, int min_rows, const int32_t* __restrict__ info) {
  if (info[0]) return;
  const int s = blockIdx.x;
  if (s >= info[1]) return;
  const int r0 = w.sptr[s], nr = w.sptr[s + 1] - r0;
  if (nr < min_rows) return;   // frames of fewer Schur rows run on the tensor-core Gram
  const int64_t rbase = w.rptr[s];   // storage position of the frame's first Schur row
  const int m = kPgD * nr, nt = (m + kPgGT - 1) / kPgGT, T = nt * (nt + 1) / 2;
  const int64_t HWs = row_stride(HW);
  __shared__ __align__(16) float Xs[kPgGK][kPgGT + 4];
  __shared__ __align__(16) float Ys[kPgGK][kPgGT + 4];
  const int tid = threadIdx.x, ty = tid >> 3, tx = tid & 7;
  const int pc = tid & 31, rh = tid >> 5;
  const float* Q = qbuf + (int64_t)s * HW;
  for (int t = blockIdx.y; t < T; t += gridDim.y) {
    int ti = 0;
    while ((ti + 1) * (ti + 2) / 2 <= t) ++ti;
    const int tj = t - ti * (ti + 1) / 2;
    // plane offsets of the 16 rows this thread stages for each side (-1: past the last row)
    int64_t ox[16], oy[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      const int x = kPgGT * ti + rh + 2 * q, y = kPgGT * tj + rh + 2 * q;
      ox[q] = x < m ? ((rbase + x / kPgD) * kPgD + x % kPgD) * HWs : -1;
      oy[q] = y < m ? ((rbase + y / kPgD) * kPgD + y % kPgD) * HWs : -1;
    }
    float acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[i][j] = 0.f;
    for (int p0 = 0; p0 < HW; p0 += kPgGK) {
      const int p = p0 + pc;
      const bool ok = p < HW;
      const float qv = ok ? Q[p] : 0.f;
      __syncthreads();
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        Xs[pc][rh + 2 * q] = (ok && ox[q] >= 0) ? erows[ox[q] + p] * qv : 0.f;
        Ys[pc][rh + 2 * q] = (ok && oy[q] >= 0) ? erows[oy[q] + p] : 0.f;
      }
      __syncthreads();
#pragma unroll 8
      for (int k = 0; k < kPgGK; ++k) {
        const float4 a = *reinterpret_cast<const float4*>(&Xs[k][4 * ty]);
        const float4 b = *reinterpret_cast<const float4*>(&Ys[k][4 * tx]);
        const float av[4] = {a.x, a.y, a.z, a.w}, bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
      }
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int x = kPgGT * ti + 4 * ty + i, y = kPgGT * tj + 4 * tx + j;
        if (x >= m || y >= m || (ti == tj && x < y)) continue;
        const double g = (double)acc[i][j];
        const int64_t pa = w.spose[r0 + x / kPgD], pb = w.spose[r0 + y / kPgD];
        const int64_t gx = 7 * pa + x % kPgD, gy = 7 * pb + y % kPgD;
        if (x == y) atomicAdd(&A[gx * npad + gy], -g);
        else if (gx > gy) atomicAdd(&A[gx * npad + gy], -g);
        else if (gy > gx) atomicAdd(&A[gy * npad + gx], -g);
        else atomicAdd(&A[gx * npad + gy], -2.0 * g);
      }
  }
}

// b -= E.(Q w) for every Schur row (Ev6x1 :1525-1560); one warp per (row, plane).
__global__ void __launch_bounds__(256)
pg_schur_rhs_kernel(int HW, BaPtrs w, const float* __restrict__ erows, const float* __restrict__ qbuf,
                    const float* __restrict__ wbuf, double* __restrict__ b, int min_rows,
                    const int32_t* __restrict__ info) {
  if (info[0]) return;
  const int s = blockIdx.x;
  if (s >= info[1]) return;
  const int r0 = w.sptr[s], nr = w.sptr[s + 1] - r0;
  if (nr < min_rows) return;
  const size_t HWs = (size_t)row_stride(HW);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const float* Q = qbuf + (int64_t)s * HW;
  const float* Wv = wbuf + (int64_t)s * HW;
  for (int task = warp; task < nr * kPgD; task += 8) {
    const int a = task / kPgD, d = task % kPgD;
    const float* e = erows + ((size_t)(w.rptr[s] + a) * kPgD + d) * HWs;
    float acc = 0.f;
    for (int p = lane; p < HW; p += 32) acc += e[p] * (Q[p] * Wv[p]);
    acc = warp_sum(acc);
    if (lane == 0) atomicAdd(&b[7 * (int64_t)w.spose[r0 + a] + d], -(double)acc);
  }
}

// dz = Q (w - sum_rows E.dx[pose]) over the frame's rows whose pose index lies in
// (0, P) (EvT6x1_kernel :1562-1582 skips ix <= 0), disps[kx] += dz (:1398-1411).
__global__ void __launch_bounds__(kPgBsThreads)
pg_backsub_kernel(float* __restrict__ disps, int HW, int P, BaPtrs w, const float* __restrict__ erows,
                  const float* __restrict__ qbuf, const float* __restrict__ wbuf, const float* __restrict__ dx,
                  float* __restrict__ dz, const int32_t* __restrict__ info) {
  if (info[0]) return;
  const int s = blockIdx.x;
  if (s >= info[1]) return;
  const size_t HWs = (size_t)row_stride(HW);
  const int r0 = w.rptr[s], r1 = w.rptr[s + 1];
  const int f = w.kx[s];
  const int base = blockIdx.y * kPgChunk + threadIdx.x;
#pragma unroll
  for (int k = 0; k < kPgBsPPT; ++k) {
    const int p = base + k * kPgBsThreads;
    if (p >= HW) continue;
    float acc = 0.f;
    for (int r = r0; r < r1; ++r) {
      const int pose = w.rpose[r];
      if (pose <= 0 || pose >= P) continue;
      const float* e = erows + (size_t)r * kPgD * HWs + p;
      float dw = 0.f;
#pragma unroll
      for (int d = 0; d < kPgD; ++d) dw += e[d * HWs] * dx[7 * pose + d];
      acc += dw;
    }
    const float v = qbuf[(int64_t)s * HW + p] * (wbuf[(int64_t)s * HW + p] - acc);
    dz[(int64_t)s * HW + p] = v;
    disps[(int64_t)f * HW + p] += v;
  }
}

struct PgLayout {
  BaLayout k;   // key arrays (the other fields are unused)
  size_t ptab, L64, hedge, erows, qbuf, wbuf, A, b, x, dxf, L11, dinv, ychol, ctl, total;
};

static PgLayout pg_layout(int64_t K, int HW, int64_t E, int P) {
  PgLayout L;
  std::memset(&L, 0, sizeof(L));
  const int64_t R = P + E;
  const int64_t S = std::min<int64_t>(K, R);
  const int64_t n = pg_order(P);
  const int64_t nbk = (n + kNB - 1) / kNB;
  size_t o = 0;
  auto take = [&](size_t bytes) { size_t at = o; o = align256(o + bytes); return at; };
  L.k.flag = take(sizeof(int) * (K + 1));
  L.k.slot = take(sizeof(int) * (K + 1));
  L.k.kx = take(sizeof(int) * (S + 1));
  L.k.gptr = take(sizeof(int) * (S + 2));
  L.k.gedge = take(sizeof(int) * (E + 1));
  L.k.cursor = take(sizeof(int) * (S + 1));
  L.k.rptr = take(sizeof(int) * (S + 2));
  L.k.rrow = take(sizeof(int) * (R + 1));
  L.k.rpose = take(sizeof(int) * (R + 1));
  L.k.sptr = take(sizeof(int) * (S + 2));
  L.k.srow = take(sizeof(int) * (R + 1));
  L.k.spose = take(sizeof(int) * (R + 1));
  L.k.epos = take(sizeof(int) * (E + 1));
  L.k.wpos = take(sizeof(int) * (P + 1));
  L.ptab = take(sizeof(float) * kPgTab * (E + 1));
  L.L64 = take(sizeof(double) * 49 * (E + 1));
  L.hedge = take(sizeof(double) * kPgH * (E + 1));
  L.erows = take(sizeof(float) * kPgD * (size_t)R * row_stride(HW));
  L.qbuf = take(sizeof(float) * (size_t)S * HW);
  L.wbuf = take(sizeof(float) * (size_t)S * HW);
  L.A = take(sizeof(double) * (size_t)(n * n + 1));
  L.b = take(sizeof(double) * (size_t)(n + 1));
  L.x = take(sizeof(double) * (size_t)(n + 1));
  L.dxf = take(sizeof(float) * (size_t)(n + 1));
  L.L11 = take(sizeof(double) * (size_t)nbk * kNB * kNB);
  L.dinv = take(sizeof(double) * (size_t)nbk * kNB);
  L.ychol = take(sizeof(double) * (size_t)(n + 1));
  L.ctl = take(sizeof(unsigned) * (4 + 3 * (size_t)nbk + (size_t)nbk * nbk));
  L.total = o;
  return L;
}

}  // namespace hs2

extern "C" int hs2_pgba_workspace_size(int64_t num_poses, int64_t num_disps, int ht, int wd, int64_t num_edges,
                                       int t0, int t1, size_t* bytes) {
  using namespace hs2;
  if (!bytes) {
    set_error("pgba_workspace_size: null output");
    return HS2_ERR_INVALID;
  }
  BaProblem p = make_problem(num_poses, num_disps, ht, wd, num_edges, t0, t1, 0);
  int rc = ba_check(p, "pgba_workspace_size");
  if (rc) return rc;
  *bytes = pg_layout(p.K, p.HW, p.E, p.P).total;
  return HS2_OK;
}

extern "C" int hs2_pgba(const float* poses, int64_t num_poses, float* disps, int64_t num_disps, int ht, int wd,
                        const float* intrinsics, const float* targets, const float* weights, const float* eta,
                        int64_t eta_rows, const float* Hsp, const float* vsp, const int64_t* iip,
                        const int64_t* jjp, int64_t num_factors, const int64_t* ii, const int64_t* jj,
                        int64_t num_edges, int t0, int t1, float lm, float ep, float* dx, float* dz,
                        int64_t dz_rows, int32_t* info, void* workspace, size_t workspace_bytes,
                        hs2_stream_t stream) {
  using namespace hs2;
  BaProblem p = make_problem(num_poses, num_disps, ht, wd, num_edges, t0, t1, 0);
  int rc = ba_check(p, "pgba");
  if (rc) return rc;
  const int P = p.P;
  const int64_t S = std::min<int64_t>(p.K, (int64_t)P + p.E);
  if (eta_rows <= 0) {
    set_error("pgba: eta must have at least one row");
    return HS2_ERR_INVALID;
  }
  if (num_factors < 0 || num_factors > (1 << 24) || (num_factors > 0 && (!Hsp || !vsp || !iip || !jjp))) {
    set_error("pgba: bad relative-pose factors (count %lld)", (long long)num_factors);
    return HS2_ERR_INVALID;
  }
  if (dz_rows < S) {
    set_error("pgba: dz needs at least %lld rows (got %lld)", (long long)S, (long long)dz_rows);
    return HS2_ERR_INVALID;
  }
  const PgLayout L = pg_layout(p.K, p.HW, p.E, P);
  if (!workspace || workspace_bytes < L.total) {
    set_error("pgba: workspace of %zu bytes required (got %zu)", L.total, workspace_bytes);
    return HS2_ERR_WORKSPACE;
  }
  if ((rc = bind_device(disps))) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  char* wsb = static_cast<char*>(workspace);
  BaPtrs w = ba_ptrs(workspace, L.k);
  float* ptab = (float*)(wsb + L.ptab);
  double* L64 = (double*)(wsb + L.L64);
  double* hedge = (double*)(wsb + L.hedge);
  float* erows = (float*)(wsb + L.erows);
  float* qbuf = (float*)(wsb + L.qbuf);
  float* wbuf = (float*)(wsb + L.wbuf);
  float* dxf = (float*)(wsb + L.dxf);
  w.A = (double*)(wsb + L.A);
  w.b = (double*)(wsb + L.b);
  w.x = (double*)(wsb + L.x);
  CholBuf cb{(double*)(wsb + L.L11), (double*)(wsb + L.dinv), (double*)(wsb + L.ychol), (unsigned*)(wsb + L.ctl)};
  const int E = (int)p.E;
  const int64_t n = 7 * (int64_t)P, npad = pg_order(P);
  const int nchunk = (p.HW + kPgChunk - 1) / kPgChunk;

  if ((rc = run_keys(p, ii, jj, eta_rows, w, info, s))) return rc;
  if (E > 0) {
    HS2_PROF("pg_edge", s);
    pg_edge_kernel<<<(7 * E + 127) / 128, 128, 0, s>>>(poses, ii, jj, E, ptab, L64, info);
    HS2_LAUNCH_CHECK("pg_edge_kernel");
    HS2_CUDA(cudaMemsetAsync(hedge, 0, sizeof(double) * kPgH * (size_t)E, s));
  }
  if (P > 0) {
    HS2_CUDA(cudaMemsetAsync(w.A, 0, sizeof(double) * (size_t)(npad * npad), s));
    HS2_CUDA(cudaMemsetAsync(w.b, 0, sizeof(double) * (size_t)npad, s));
    pg_pad_kernel<<<1, 32, 0, s>>>(w.A, n, npad);
    HS2_LAUNCH_CHECK("pg_pad_kernel");
  }
  if (S > 0) {
    HS2_PROF("pg_linearize", s);
    pg_linearize_kernel<<<dim3((unsigned)S, nchunk), kPgThreads, 0, s>>>(
        disps, p.HW, p.wd, intrinsics, targets, weights, eta, eta_rows, jj, t0, t1, ptab, w, erows, qbuf, wbuf, hedge,
        info);
    HS2_LAUNCH_CHECK("pg_linearize_kernel");
  }
  if (E > 0 && P > 0) {
    HS2_PROF("pg_assemble", s);
    pg_assemble_kernel<<<(7 * E + 127) / 128, 128, 0, s>>>(ii, jj, E, t0, npad, L64, hedge, w.A, w.b, info);
    HS2_LAUNCH_CHECK("pg_assemble_kernel");
  }
  if (num_factors > 0) {
    HS2_PROF("pg_prior", s);
    pg_prior_kernel<<<(unsigned)((7 * num_factors + 127) / 128), 128, 0, s>>>(Hsp, vsp, iip, jjp, num_factors, t0,
                                                                              t1, npad, w.A, w.b, info);
    HS2_LAUNCH_CHECK("pg_prior_kernel");
  }
  if (P > 0 && S > 0) {
    HS2_PROF("pg_schur", s);
    // frames of <= 36 Schur rows (N = 7 R + 1 <= 256): the tensor-core Gram of ba with
    // 7-value rows, its w row giving the rhs; larger frames: the SIMT Gram + rhs kernels
    const bool tc = g_schur_path.load() == 0;
    if (tc) {
      static DeviceOnce once;
      int dev = 0;
      HS2_CUDA(cudaGetDevice(&dev));
      rc = once.run(dev, [&]() -> int {
        HS2_CUDA(cudaFuncSetAttribute(ba_schur_tc_kernel<7>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem));
        return HS2_OK;
      });
      if (rc) return rc;
      CUtensorMap emap;
      if ((rc = encode_erows_map(&emap, erows, p.HW, kPgD * ((int64_t)P + E)))) return rc;
      BaPtrs wt = w;
      wt.erows = erows;
      wt.qbuf = qbuf;
      wt.wbuf = wbuf;
      const BaLaunch l = ba_launch_shape(p);
      dim3 grid((unsigned)S, 1u, l.tc_split);
      ba_schur_tc_kernel<7><<<grid, kTcThreads, kTcSmem, s>>>(emap, p.HW, l.tc_chunk, wt, npad, info,
                                                              g_gram_split3.load());
      HS2_LAUNCH_CHECK("ba_schur_tc_kernel<7>");
    }
    const int min_rows = tc ? tc_max_blocks(kPgD) + 1 : 0;
    pg_schur_kernel<<<dim3((unsigned)S, kPgSplit), kPgGThreads, 0, s>>>(p.HW, npad, w, erows, qbuf, w.A, min_rows,
                                                                        info);
    HS2_LAUNCH_CHECK("pg_schur_kernel");
    pg_schur_rhs_kernel<<<(unsigned)S, 256, 0, s>>>(p.HW, w, erows, qbuf, wbuf, w.b, min_rows, info);
    HS2_LAUNCH_CHECK("pg_schur_rhs_kernel");
  }
  if (P > 0) {
    if ((rc = run_cholesky((int)npad, lm, ep, w, cb, dxf, info, s))) return rc;
    HS2_CUDA(cudaMemcpyAsync(dx, dxf, sizeof(float) * (size_t)n, cudaMemcpyDeviceToDevice, s));
  }
  if (S > 0) {
    HS2_PROF("pg_backsub", s);
    pg_backsub_kernel<<<dim3((unsigned)S, nchunk), kPgBsThreads, 0, s>>>(disps, p.HW, P, w, erows, qbuf, wbuf, dxf,
                                                                       dz, info);
    HS2_LAUNCH_CHECK("pg_backsub_kernel");
  }
  return HS2_OK;
}

#include <vector>
#include "ba_batch.cuh"
