// Workspace layout of the dense BA (one window) and the per-pixel linearisation,
// shared by the single-window kernels (ba.cu) and the batched ones (ba_batch.cu).
#pragma once

#include <algorithm>

#include "common.cuh"

namespace hs2 {

constexpr int kNB = 64;                             // blocked Cholesky tile
constexpr int kEtab = 56;                           // floats per edge in the edge table

// ------------------------------------------------------------ workspace ---
struct BaLayout {
  size_t flag, slot, kx, gptr, gedge, cursor, rptr, rrow, rpose, sptr, srow, spose, epos, wpos;
  size_t etab, etab64, hedge, erows, qbuf, wbuf, A, b, x, chol_fail, L11, dinv, ychol, ctl, total;
};

static size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Row stride (floats) of the E-row planes: pixels padded to 32 so that every plane
// row starts on a 128-byte boundary (TMA tiles of 32 pixels).
static __host__ __device__ __forceinline__ int row_stride(int HW) { return (HW + 31) & ~31; }

static BaLayout ba_layout(int64_t K, int HW, int64_t E, int P, int motion_only) {
  BaLayout L;
  const int64_t R = P + E;
  const int64_t S = std::min<int64_t>(K, R);  // depth-slot capacity
  const int64_t n = 6 * (int64_t)P;
  size_t o = 0;
  auto take = [&](size_t bytes) { size_t at = o; o = align256(o + bytes); return at; };
  L.flag = take(sizeof(int) * (K + 1));
  L.slot = take(sizeof(int) * (K + 1));
  L.kx = take(sizeof(int) * (S + 1));
  L.gptr = take(sizeof(int) * (S + 2));
  L.gedge = take(sizeof(int) * (E + 1));
  L.cursor = take(sizeof(int) * (S + 1));
  L.rptr = take(sizeof(int) * (S + 2));
  L.rrow = take(sizeof(int) * (R + 1));
  L.rpose = take(sizeof(int) * (R + 1));
  L.sptr = take(sizeof(int) * (S + 2));
  L.srow = take(sizeof(int) * (R + 1));
  L.spose = take(sizeof(int) * (R + 1));
  L.epos = take(sizeof(int) * (E + 1));
  L.wpos = take(sizeof(int) * (P + 1));
  L.etab = take(sizeof(float) * kEtab * (E + 1));
  L.etab64 = take(sizeof(double) * 36 * (E + 1));
  L.hedge = take(sizeof(double) * 27 * (E + 1));
  L.erows = take(motion_only ? 0 : sizeof(float) * 6 * (size_t)R * row_stride(HW));
  L.qbuf = take(motion_only ? 0 : sizeof(float) * (size_t)S * HW);
  L.wbuf = take(motion_only ? 0 : sizeof(float) * (size_t)S * HW);
  L.A = take(sizeof(double) * (size_t)(n * n + 1));
  L.b = take(sizeof(double) * (size_t)(n + 1));
  L.x = take(sizeof(double) * (size_t)(n + 1));
  L.chol_fail = take(sizeof(int) * 4);
  L.L11 = take(sizeof(double) * (size_t)((n + kNB - 1) / kNB) * kNB * kNB);
  L.dinv = take(sizeof(double) * (size_t)((n + kNB - 1) / kNB) * kNB);
  L.ychol = take(sizeof(double) * (size_t)(n + 1));
  L.ctl = take(sizeof(unsigned) * (4 + 3 * (size_t)((n + kNB - 1) / kNB) +
                                    (size_t)((n + kNB - 1) / kNB) * ((n + kNB - 1) / kNB)));   // see CholBuf
  L.total = o;
  return L;
}

struct BaPtrs {
  int *flag, *slot, *kx, *gptr, *gedge, *cursor, *rptr, *rrow, *rpose, *sptr, *srow, *spose, *epos, *wpos;
  float* etab;
  double *etab64, *hedge;
  float *erows, *qbuf, *wbuf;
  double *A, *b, *x;
  int* chol_fail;
};

static BaPtrs ba_ptrs(void* ws, const BaLayout& L) {
  char* base = static_cast<char*>(ws);
  BaPtrs p;
  p.flag = (int*)(base + L.flag);
  p.slot = (int*)(base + L.slot);
  p.kx = (int*)(base + L.kx);
  p.gptr = (int*)(base + L.gptr);
  p.gedge = (int*)(base + L.gedge);
  p.cursor = (int*)(base + L.cursor);
  p.rptr = (int*)(base + L.rptr);
  p.rrow = (int*)(base + L.rrow);
  p.rpose = (int*)(base + L.rpose);
  p.sptr = (int*)(base + L.sptr);
  p.srow = (int*)(base + L.srow);
  p.spose = (int*)(base + L.spose);
  p.epos = (int*)(base + L.epos);
  p.wpos = (int*)(base + L.wpos);
  p.etab = (float*)(base + L.etab);
  p.etab64 = (double*)(base + L.etab64);
  p.hedge = (double*)(base + L.hedge);
  p.erows = (float*)(base + L.erows);
  p.qbuf = (float*)(base + L.qbuf);
  p.wbuf = (float*)(base + L.wbuf);
  p.A = (double*)(base + L.A);
  p.b = (double*)(base + L.b);
  p.x = (double*)(base + L.x);
  p.chol_fail = (int*)(base + L.chol_fail);
  return p;
}


// Upper-triangle order of the 21 entries of a symmetric 6x6 block.
__device__ __forceinline__ int tri6(int r, int c) { return r * 6 - (r * (r - 1)) / 2 + (c - r); }

// Linearisation of one pixel for one edge (reference projective_transform and the
// per-pixel part of projective_transform_kernel): the point of normalised image
// coordinates (xn, yn) at disparity h is moved by Gij (tab: t at 0..2, rotation matrix
// at 44..52) and projected.  Outputs the point Jacobian products of the edge's
// Hessian block (27 sums: upper triangle of Hjj, then vj) added to H, the Schur
// terms C (cs) and w (ws), and the row E_j (6).  Pixels closer than kMinDepth
// contribute nothing but their (zero-weight) residual; a self edge keeps C and w and
// drops H and E.  The Jacobians have a structural zero each (Ju[1], Jv[0]): those
// products are never formed.
__device__ __forceinline__ void lin_pixel(const float* __restrict__ tab, float fx, float fy, float cx, float cy,
                                          float xn, float yn, float h, float tu, float tv, float wgu, float wgv,
                                          bool self, float (&H)[32], float& cs, float& ws, float (&Ej)[6]) {
  const float* R = tab + 44;
  const float Y0 = fmaf(R[0], xn, fmaf(R[1], yn, R[2])) + h * tab[0];
  const float Y1 = fmaf(R[3], xn, fmaf(R[4], yn, R[5])) + h * tab[1];
  const float Y2 = fmaf(R[6], xn, fmaf(R[7], yn, R[8])) + h * tab[2];
  const bool bad = Y2 < kMinDepth;
  const float iz = __fdividef(1.0f, Y2);
  const float xp = fx * (Y0 * iz) + cx;
  const float yp = fy * (Y1 * iz) + cy;
  const float z = bad ? 0.f : Y2;
  const float dd = bad ? 0.f : iz;
  const float d2 = dd * dd;
  float wu = bad ? 0.f : 0.001f * wgu;
  float wv = bad ? 0.f : 0.001f * wgv;
  const float ru = tu - xp, rv = tv - yp;
  const float Jp0 = fx * dd, Jp2 = fx * (-Y0 * d2);
  const float Jp4 = fy * dd, Jp5 = fy * (-Y1 * d2);
  const float Ju[6] = {Jp0 * h, 0.f, Jp2 * h, Jp2 * Y1, Jp0 * z - Jp2 * Y0, -Jp0 * Y1};
  const float Jv[6] = {0.f, Jp4 * h, Jp5 * h, -Jp4 * z + Jp5 * Y1, -Jp5 * Y0, Jp4 * Y0};
  const float Jzu = Jp0 * tab[0] + Jp2 * tab[2];
  const float Jzv = Jp4 * tab[1] + Jp5 * tab[2];
  cs += wu * Jzu * Jzu + wv * Jzv * Jzv;
  ws += wu * ru * Jzu + wv * rv * Jzv;
  if (self) { wu = 0.f; wv = 0.f; }
  const float au = wu * ru, av = wv * rv;
#pragma unroll
  for (int r = 0; r < 6; ++r) {
    const float su = wu * Ju[r], sv = wv * Jv[r];
#pragma unroll
    for (int c = r; c < 6; ++c) {
      if (r != 1 && c != 1) H[tri6(r, c)] = fmaf(su, Ju[c], H[tri6(r, c)]);
      if (r != 0 && c != 0) H[tri6(r, c)] = fmaf(sv, Jv[c], H[tri6(r, c)]);
    }
    if (r != 1) H[21 + r] = fmaf(au, Ju[r], H[21 + r]);
    if (r != 0) H[21 + r] = fmaf(av, Jv[r], H[21 + r]);
  }
  const float zu = wu * Jzu, zv = wv * Jzv;
  Ej[0] = zu * Ju[0];
  Ej[1] = zv * Jv[1];
#pragma unroll
  for (int r = 2; r < 6; ++r) Ej[r] = fmaf(zu, Ju[r], zv * Jv[r]);
}


// Keys of one window (ba.cu): depth slots, edge groups by source frame, E-row lists.
__global__ void ba_keys_kernel(const int64_t* __restrict__ ii, const int64_t* __restrict__ jj, int E, int K, int t0,
                               int t1, int64_t eta_rows, BaPtrs w, int32_t* __restrict__ info);
// Per-edge table of one window (ba.cu): Gij, its rotation matrix, the map L (Ji = L Jj).
__global__ void ba_edge_setup_kernel(const float* __restrict__ poses, const int64_t* __restrict__ ii,
                                     const int64_t* __restrict__ jj, int E, float* __restrict__ etab,
                                     double* __restrict__ etab64, const int32_t* __restrict__ info);

}  // namespace hs2
