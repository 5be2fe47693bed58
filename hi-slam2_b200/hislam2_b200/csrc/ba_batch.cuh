// Batched bundle adjustment: many independent windows (uneven keyframe and edge
// counts, grids of different sizes) in ONE persistent launch per Levenberg-Marquardt
// iteration.  Included at the end of ba.cu: the work units run the same device
// bodies as the single-window kernels.
//
// Work units, handed out phase-major by an atomic counter (every unit of phase k of
// every window before any unit of phase k+1):
//   0  edge table (ba_edge_setup) in 256-edge-thread units, + one unit zeroing the
//      window's per-edge sums and FP64 system;
//   1  linearisation, one unit per (depth frame, 1024 pixels) (ba_linearize body,
//      256 threads);
//   2  assembly (256 edge threads per unit) and the SIMT Schur Gram, one unit per
//      (depth frame, pixel split) (ba_schur body);
//   3  the damped FP64 Cholesky solve of the window's reduced system, one unit
//      (single CTA: 32-column panels in shared memory for systems up to 256 wide,
//      column by column in global memory above that, up to 6 * kBatchMaxPoses);
//   4  back-substitution per (depth frame, 1024 pixels) and the pose retraction.
// A unit of phase k > 0 waits (acquire, bounded) until the window's phase k-1
// counter reaches its unit count; units count themselves done with a release add.
// Every unit of an earlier phase was handed to a resident CTA before the wait
// begins (cooperative launch: all CTAs co-resident), so no wait can cycle.  A wait
// that runs out sets HS2_DEV_TIMEOUT in the window's info and the launch drains.
// The keys (depth slots, edge groups, E-row lists) do not change between
// iterations and are built once by hs2_ba_batch_prepare.
namespace hs2 {

constexpr int kBatchThreads = 256;
constexpr int kBatchPhases = 5;
constexpr int kBatchMaxPoses = 256;     // 6 * 256 = 1536-wide reduced systems at most
constexpr unsigned kBatchSpin = 1u << 24;

// Test hooks for the bounded waits (hs2_ba_batch_set_wait_test): the number of polls
// a dependency wait makes before it gives up, and a switch that adds one to every
// count a wait needs, so that no wait can be satisfied and each one runs out.
__device__ unsigned g_batch_spin = kBatchSpin;
__device__ unsigned g_batch_unsatisfiable = 0;

struct BatchWin {
  float* poses;
  float* disps;
  const float* intr;
  const float* targets;
  const float* weights;
  const float* eta;
  const int64_t* ii;
  const int64_t* jj;
  float* dx;
  float* dz;
  int32_t* info;
  int64_t K, E, eta_rows, dz_rows;
  int HW, wd, t0, t1, P, S;
  int nsetup, nlin, nasm, gsplit, gchunk, nback;
  int units[kBatchPhases];
  BaPtrs w;
};

struct BatchHdr {
  int nwin;
  int total;                          // units of all phases
  int cum[kBatchPhases + 1];          // first unit of each phase
  int grid;                           // CTAs of the persistent launch
};

// Damped FP64 Cholesky of the lower triangle of A (n x n, row-major) and the solve
// A x = b, by one CTA; x lands in w.x (double) and dx (float).  A pivot that is not
// positive leaves x = 0 and counts a failed factorisation in info[2] (the
// reference's SimplicialLLT failure gives a zero update, droid_kernels.cu:1666-1677).
__device__ void batch_cholesky_solve(int n, float lm, float ep, BaPtrs w, float* __restrict__ dx,
                                     int32_t* __restrict__ info) {
  double* A = w.A;
  double* y = w.b;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  __shared__ double piv;
  __shared__ int failed;
  if (tid == 0) failed = 0;
  for (int i = tid; i < n; i += kBatchThreads) {
    const double d = A[(int64_t)i * n + i];
    A[(int64_t)i * n + i] = d + (ep + lm * d);
  }
  __syncthreads();
  for (int k = 0; k < n; ++k) {
    if (tid == 0) {
      const double d = A[(int64_t)k * n + k];
      if (!(d > 0.0)) failed = 1;
      else {
        piv = sqrt(d);
        A[(int64_t)k * n + k] = piv;
      }
    }
    __syncthreads();
    if (failed) break;
    const double inv = 1.0 / piv;
    for (int i = k + 1 + tid; i < n; i += kBatchThreads) A[(int64_t)i * n + k] *= inv;
    __syncthreads();
    for (int i = k + 1 + warp; i < n; i += kBatchThreads / 32) {
      const double lik = A[(int64_t)i * n + k];
      for (int j = k + 1 + lane; j <= i; j += 32) A[(int64_t)i * n + j] -= lik * A[(int64_t)j * n + k];
    }
    __syncthreads();
  }
  if (failed) {
    for (int i = tid; i < n; i += kBatchThreads) {
      w.x[i] = 0.0;
      dx[i] = 0.f;
    }
    if (tid == 0) atomicAdd(&info[2], 1);
    return;
  }
  // L y = b (column order), then L^T x = y, in place in w.b
  for (int k = 0; k < n; ++k) {
    if (tid == 0) y[k] /= A[(int64_t)k * n + k];
    __syncthreads();
    const double yk = y[k];
    for (int i = k + 1 + tid; i < n; i += kBatchThreads) y[i] -= A[(int64_t)i * n + k] * yk;
    __syncthreads();
  }
  for (int k = n - 1; k >= 0; --k) {
    if (tid == 0) y[k] /= A[(int64_t)k * n + k];
    __syncthreads();
    const double xk = y[k];
    for (int i = tid; i < k; i += kBatchThreads) y[i] -= A[(int64_t)k * n + i] * xk;
    __syncthreads();
  }
  for (int i = tid; i < n; i += kBatchThreads) {
    w.x[i] = y[i];
    dx[i] = (float)y[i];
  }
}

// Blocked form of the same factorisation and solve for systems of at most
// kBatchPanelRows unknowns: 32-column panels are factored in shared memory (pv:
// kBatchPanelRows x 33 doubles of dynamic shared memory), the trailing matrix is
// updated with 32-long dot products against the panel, and the two triangular
// solves go block by block (diagonal block in shared memory, one warp eliminating
// its 32 unknowns, all threads applying the off-diagonal blocks).  Same results as
// batch_cholesky_solve up to rounding; same failure rule.
constexpr int kBatchPanelRows = 256;
constexpr int kBatchPanelLd = 33;
constexpr size_t kBatchDynSmem = sizeof(double) * kBatchPanelRows * kBatchPanelLd;

__device__ void batch_cholesky_blocked(int n, float lm, float ep, BaPtrs w, float* __restrict__ dx,
                                       int32_t* __restrict__ info, double* __restrict__ pv) {
  double* A = w.A;
  double* y = w.b;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int NW = kBatchThreads / 32;
  __shared__ int failed;
  __shared__ double red[NW][32];
  if (tid == 0) failed = 0;
  for (int i = tid; i < n; i += kBatchThreads) {
    const double d = A[(int64_t)i * n + i];
    A[(int64_t)i * n + i] = d + (ep + lm * d);
  }
  __syncthreads();
  for (int kb = 0; kb < n; kb += 32) {
    const int nc = min(32, n - kb), rows = n - kb;
    for (int i = warp; i < rows; i += NW)
      for (int c = lane; c < nc; c += 32) pv[i * kBatchPanelLd + c] = c <= i ? A[(int64_t)(kb + i) * n + kb + c] : 0.0;
    __syncthreads();
    for (int c = 0; c < nc; ++c) {
      if (tid == 0) {
        const double d = pv[c * kBatchPanelLd + c];
        if (!(d > 0.0)) failed = 1;
        else pv[c * kBatchPanelLd + c] = sqrt(d);
      }
      __syncthreads();
      if (failed) break;
      const double inv = 1.0 / pv[c * kBatchPanelLd + c];
      for (int i = c + 1 + tid; i < rows; i += kBatchThreads) pv[i * kBatchPanelLd + c] *= inv;
      __syncthreads();
      // rank-1 update of the panel's remaining columns (c2 <= i)
      for (int i = c + 1 + warp; i < rows; i += NW) {
        const double lic = pv[i * kBatchPanelLd + c];
        for (int c2 = c + 1 + lane; c2 < nc && c2 <= i; c2 += 32)
          pv[i * kBatchPanelLd + c2] -= lic * pv[c2 * kBatchPanelLd + c];
      }
      __syncthreads();
    }
    if (failed) break;
    for (int i = warp; i < rows; i += NW)
      for (int c = lane; c < nc; c += 32)
        if (c <= i) A[(int64_t)(kb + i) * n + kb + c] = pv[i * kBatchPanelLd + c];
    // trailing update A[i][j] -= L[i, panel] . L[j, panel] for kb + nc <= j <= i
    for (int i = nc + warp; i < rows; i += NW) {
      const double* li = pv + i * kBatchPanelLd;
      for (int j = nc + lane; j <= i; j += 32) {
        const double* lj = pv + j * kBatchPanelLd;
        double acc = 0.0;
#pragma unroll 8
        for (int c = 0; c < nc; ++c) acc = fma(li[c], lj[c], acc);
        A[(int64_t)(kb + i) * n + kb + j] -= acc;
      }
    }
    __syncthreads();
  }
  if (failed) {
    for (int i = tid; i < n; i += kBatchThreads) {
      w.x[i] = 0.0;
      dx[i] = 0.f;
    }
    if (tid == 0) atomicAdd(&info[2], 1);
    return;
  }
  // forward L y = b, block by block (y in place in w.b)
  for (int kb = 0; kb < n; kb += 32) {
    const int nc = min(32, n - kb);
    for (int i = warp; i < nc; i += NW)
      for (int c = lane; c <= i; c += 32) pv[i * kBatchPanelLd + c] = A[(int64_t)(kb + i) * n + kb + c];
    __syncthreads();
    if (warp == 0) {
      double yc = lane < nc ? y[kb + lane] : 0.0;
      for (int k = 0; k < nc; ++k) {
        if (lane == k) yc /= pv[k * kBatchPanelLd + k];
        const double yk = __shfl_sync(0xffffffffu, yc, k);
        if (lane > k && lane < nc) yc -= pv[lane * kBatchPanelLd + k] * yk;
      }
      if (lane < nc) y[kb + lane] = yc;
    }
    __syncthreads();
    for (int i = kb + nc + tid; i < n; i += kBatchThreads) {
      double acc = 0.0;
      for (int c = 0; c < nc; ++c) acc = fma(A[(int64_t)i * n + kb + c], y[kb + c], acc);
      y[i] -= acc;
    }
    __syncthreads();
  }
  // backward L^T x = y, last block first
  const int nblk = (n + 31) / 32;
  for (int bk = nblk - 1; bk >= 0; --bk) {
    const int kb = bk * 32, nc = min(32, n - kb);
    // y[kb + c] -= sum_{i >= kb + nc} L[i][kb + c] x[i]
    double part = 0.0;
    if (lane < nc)
      for (int i = kb + nc + warp; i < n; i += NW) part = fma(A[(int64_t)i * n + kb + lane], y[i], part);
    red[warp][lane] = part;
    for (int i = warp; i < nc; i += NW)
      for (int c = lane; c <= i; c += 32) pv[i * kBatchPanelLd + c] = A[(int64_t)(kb + i) * n + kb + c];
    __syncthreads();
    if (warp == 0) {
      double yc = 0.0;
      if (lane < nc) {
        double t = 0.0;
        for (int k = 0; k < NW; ++k) t += red[k][lane];
        yc = y[kb + lane] - t;
      }
      for (int k = nc - 1; k >= 0; --k) {
        if (lane == k) yc /= pv[k * kBatchPanelLd + k];
        const double xk = __shfl_sync(0xffffffffu, yc, k);
        if (lane < k) yc -= pv[k * kBatchPanelLd + lane] * xk;
      }
      if (lane < nc) y[kb + lane] = yc;
    }
    __syncthreads();
  }
  for (int i = tid; i < n; i += kBatchThreads) {
    w.x[i] = y[i];
    dx[i] = (float)y[i];
  }
}

__device__ void batch_unit(const BatchWin& W, int ph, int idx, float lm, float ep, double* pv) {
  const int tid = threadIdx.x;
  const BaPtrs& w = W.w;
  const int n = 6 * W.P;
  switch (ph) {
    case 0:
      if (idx < W.nsetup) {
        if (W.info[0] == 0) ba_edge_setup_body(idx * kBatchThreads + tid, W.poses, W.ii, W.jj, (int)W.E, w.etab,
                                               w.etab64, W.info);
      } else {
        for (int64_t i = tid; i < 27 * W.E; i += kBatchThreads) w.hedge[i] = 0.0;
        for (int64_t i = tid; i < (int64_t)n * n; i += kBatchThreads) w.A[i] = 0.0;
        for (int i = tid; i < n; i += kBatchThreads) w.b[i] = 0.0;
      }
      break;
    case 1:
      ba_linearize_body<kBatchThreads>(idx / W.nlin, idx % W.nlin, W.disps, W.HW, W.wd, W.intr, W.targets,
                                       W.weights, W.eta, W.eta_rows, W.jj, W.t0, W.t1, 0, 0, w, W.info);
      break;
    case 2:
      if (idx < W.nasm) {
        ba_assemble_body(idx * kBatchThreads + tid, W.ii, W.jj, (int)W.E, W.t0, W.P, w, W.info);
      } else {
        const int g = idx - W.nasm;
        ba_schur_body(g / W.gsplit, g % W.gsplit, W.HW, W.gchunk, w, W.P, 1, 0, W.info);
      }
      break;
    case 3:
      if (W.info[0] == 0 && n > 0) {
        if (n <= kBatchPanelRows) batch_cholesky_blocked(n, lm, ep, w, W.dx, W.info, pv);
        else batch_cholesky_solve(n, lm, ep, w, W.dx, W.info);
      }
      break;
    default:
      if (idx < W.nback) {
        ba_backsub_body<kBatchThreads>(idx / W.nlin, idx % W.nlin, W.disps, W.HW, W.P, w, W.dx, W.dz, W.dz_rows,
                                       W.info);
      } else {
        for (int k = tid; k < W.P; k += kBatchThreads) ba_pose_retr_body(k, W.poses, W.t0, W.P, w, W.info);
      }
      break;
  }
}

__global__ void __launch_bounds__(kBatchThreads, 2)
ba_batch_kernel(const BatchHdr* __restrict__ hdr, const BatchWin* __restrict__ wins, const int* __restrict__ prefix,
                unsigned* __restrict__ done, unsigned* __restrict__ next, int* __restrict__ abort_flag, float lm,
                float ep) {
  __shared__ int s_u, s_ph, s_w, s_idx, s_go;
  extern __shared__ double batch_dyn[];       // the blocked Cholesky's panel
  const int nwin = hdr->nwin, total = hdr->total;
  for (;;) {
    if (threadIdx.x == 0) {
      const int u = (int)atomicAdd(next, 1u);
      s_u = u;
      if (u < total) {
        int ph = 0;
        while (u >= hdr->cum[ph + 1]) ++ph;
        const int local = u - hdr->cum[ph];
        const int* pre = prefix + ph * (nwin + 1);
        int lo = 0, hi = nwin - 1;          // last window with pre[w] <= local
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (pre[mid] <= local) lo = mid;
          else hi = mid - 1;
        }
        s_ph = ph;
        s_w = lo;
        s_idx = local - pre[lo];
        int go = 1;
        if (ph > 0) {
          const unsigned need = (unsigned)wins[lo].units[ph - 1] + g_batch_unsatisfiable;
          const unsigned limit = g_batch_spin;
          const unsigned* c = done + lo * kBatchPhases + ph - 1;
          unsigned i = 0;
          while (ld_acquire_gpu(c) < need) {
            if (++i > limit || *(volatile int*)abort_flag) {
              // only the launch-wide flag is raised here: the bodies of other CTAs read the
              // windows' info words, which therefore must not change during the launch
              go = 0;
              if (i > limit) atomicExch(abort_flag, 1);
              break;
            }
          }
        }
        s_go = go && !*(volatile int*)abort_flag;
      }
    }
    __syncthreads();
    if (s_u >= total) break;
    if (s_go) batch_unit(wins[s_w], s_ph, s_idx, lm, ep, batch_dyn);
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      red_release_add_gpu(done + s_w * kBatchPhases + s_ph, 1u);
    }
  }
}

// After a launch that gave up (a bounded wait ran out), every window's results are
// incomplete: mark them all.
__global__ void ba_batch_flag_kernel(const BatchWin* __restrict__ wins, int nwin, const int* __restrict__ abort_flag) {
  if (*abort_flag == 0) return;
  for (int k = threadIdx.x; k < nwin; k += blockDim.x) atomicOr(wins[k].info, HS2_DEV_TIMEOUT);
}

// ----------------------------------------------------------------- host ---
struct BatchPlanHost {
  BatchHdr hdr;
  std::vector<BatchWin> wins;
  std::vector<int> prefix;
  size_t off_hdr, off_wins, off_prefix, off_ctl, ctl_bytes, off_ws, total;
  std::vector<size_t> ws_off;
};

static int batch_plan(const hs2_ba_window* in, int nwin, int gsplit, BatchPlanHost& pl) {
  if (nwin <= 0 || !in) {
    set_error("ba_batch: no windows");
    return HS2_ERR_INVALID;
  }
  if (gsplit < 1 || gsplit > 64) {
    set_error("ba_batch: gram split %d outside [1, 64]", gsplit);
    return HS2_ERR_INVALID;
  }
  pl.wins.resize(nwin);
  pl.ws_off.resize(nwin);
  size_t o = 0;
  auto take = [&](size_t bytes) { size_t at = o; o = align256(o + bytes); return at; };
  pl.off_hdr = take(sizeof(BatchHdr));
  pl.off_wins = take(sizeof(BatchWin) * nwin);
  pl.off_prefix = take(sizeof(int) * kBatchPhases * (nwin + 1));
  pl.ctl_bytes = sizeof(unsigned) * (kBatchPhases * (size_t)nwin + 2);
  pl.off_ctl = take(pl.ctl_bytes);
  for (int k = 0; k < nwin; ++k) {
    const hs2_ba_window& a = in[k];
    char what[48];
    snprintf(what, sizeof(what), "ba_batch window %d", k);
    BaProblem p = make_problem(a.num_poses, a.num_disps, a.ht, a.wd, a.num_edges, a.t0, a.t1, 0);
    int rc = ba_check(p, what);
    if (rc) return rc;
    if (p.P > kBatchMaxPoses) {
      set_error("%s: %d optimised poses, the batched solver takes at most %d", what, p.P, kBatchMaxPoses);
      return HS2_ERR_INVALID;
    }
    if (!a.poses || !a.disps || !a.intrinsics || !a.info || !a.eta || (p.E > 0 && (!a.targets || !a.weights ||
        !a.ii || !a.jj)) || (p.P > 0 && !a.dx) || !a.dz) {
      set_error("%s: null pointer", what);
      return HS2_ERR_INVALID;
    }
    const BaLayout L = ba_layout(p.K, p.HW, p.E, p.P, 0);
    pl.ws_off[k] = take(L.total);
    BatchWin& W = pl.wins[k];
    W.poses = a.poses;
    W.disps = a.disps;
    W.intr = a.intrinsics;
    W.targets = a.targets;
    W.weights = a.weights;
    W.eta = a.eta;
    W.ii = a.ii;
    W.jj = a.jj;
    W.dx = a.dx;
    W.dz = a.dz;
    W.info = a.info;
    W.K = p.K;
    W.E = p.E;
    W.eta_rows = a.eta_rows;
    W.dz_rows = a.dz_rows;
    W.HW = p.HW;
    W.wd = p.wd;
    W.t0 = p.t0;
    W.t1 = p.t1;
    W.P = p.P;
    W.S = (int)std::min<int64_t>(p.K, (int64_t)p.P + p.E);
    const int chunk = kBatchThreads * kLinPPT;
    W.nlin = (p.HW + chunk - 1) / chunk;
    W.nsetup = (int)((6 * p.E + kBatchThreads - 1) / kBatchThreads);
    W.nasm = W.nsetup;
    W.gsplit = gsplit;
    W.gchunk = ((p.HW + gsplit - 1) / gsplit + kSchurTP - 1) / kSchurTP * kSchurTP;
    W.nback = W.S * W.nlin;
    W.units[0] = W.nsetup + 1;
    W.units[1] = W.S * W.nlin;
    W.units[2] = W.nasm + W.S * gsplit;
    W.units[3] = 1;
    W.units[4] = W.nback + 1;
  }
  pl.off_ws = pl.ws_off.empty() ? o : pl.ws_off[0];
  pl.total = o;
  pl.prefix.assign(kBatchPhases * (nwin + 1), 0);
  pl.hdr.nwin = nwin;
  pl.hdr.cum[0] = 0;
  for (int ph = 0; ph < kBatchPhases; ++ph) {
    int acc = 0;
    for (int k = 0; k < nwin; ++k) {
      pl.prefix[ph * (nwin + 1) + k] = acc;
      acc += pl.wins[k].units[ph];
    }
    pl.prefix[ph * (nwin + 1) + nwin] = acc;
    pl.hdr.cum[ph + 1] = pl.hdr.cum[ph] + acc;
  }
  pl.hdr.total = pl.hdr.cum[kBatchPhases];
  return HS2_OK;
}

}  // namespace hs2

extern "C" int hs2_ba_batch_workspace_size(const hs2_ba_window* windows, int num_windows, size_t* bytes) {
  using namespace hs2;
  if (!bytes) {
    set_error("ba_batch_workspace_size: null output");
    return HS2_ERR_INVALID;
  }
  BatchPlanHost pl;
  int rc = batch_plan(windows, num_windows, 1, pl);
  if (rc) return rc;
  *bytes = pl.total;
  return HS2_OK;
}

extern "C" int hs2_ba_batch_prepare(const hs2_ba_window* windows, int num_windows, int gram_split, int ctas_per_sm,
                                    void* workspace, size_t workspace_bytes, int* grid, hs2_stream_t stream) {
  using namespace hs2;
  BatchPlanHost pl;
  int rc = batch_plan(windows, num_windows, gram_split, pl);
  if (rc) return rc;
  if (!workspace || workspace_bytes < pl.total) {
    set_error("ba_batch_prepare: workspace of %zu bytes required", pl.total);
    return HS2_ERR_WORKSPACE;
  }
  if (!grid) {
    set_error("ba_batch_prepare: null grid output");
    return HS2_ERR_INVALID;
  }
  if ((rc = bind_device(workspace))) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  char* base = static_cast<char*>(workspace);
  int dev = 0, sms = 0, occ = 0;
  HS2_CUDA(cudaGetDevice(&dev));
  HS2_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  HS2_CUDA(cudaFuncSetAttribute(ba_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBatchDynSmem));
  HS2_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, ba_batch_kernel, kBatchThreads, kBatchDynSmem));
  if (occ < 1) {
    set_error("ba_batch_prepare: the batched kernel does not fit on an SM");
    return HS2_ERR_CUDA;
  }
  const int per_sm = ctas_per_sm <= 0 ? occ : std::min(ctas_per_sm, occ);
  pl.hdr.grid = std::max(1, std::min(per_sm * sms, pl.hdr.total));
  for (int k = 0; k < num_windows; ++k) pl.wins[k].w = ba_ptrs(base + pl.ws_off[k], ba_layout(pl.wins[k].K,
                                                       pl.wins[k].HW, pl.wins[k].E, pl.wins[k].P, 0));
  // the descriptor tables are copied synchronously: prepare is not meant for capture
  HS2_CUDA(cudaMemcpyAsync(base + pl.off_hdr, &pl.hdr, sizeof(BatchHdr), cudaMemcpyHostToDevice, s));
  HS2_CUDA(cudaMemcpyAsync(base + pl.off_wins, pl.wins.data(), sizeof(BatchWin) * num_windows,
                           cudaMemcpyHostToDevice, s));
  HS2_CUDA(cudaMemcpyAsync(base + pl.off_prefix, pl.prefix.data(), sizeof(int) * pl.prefix.size(),
                           cudaMemcpyHostToDevice, s));
  for (int k = 0; k < num_windows; ++k) {
    const hs2_ba_window& a = windows[k];
    const BatchWin& W = pl.wins[k];
    HS2_CUDA(cudaMemsetAsync(a.info, 0, 4 * sizeof(int32_t), s));
    HS2_PROF("ba_keys", s);
    ba_keys_kernel<<<1, 1024, 0, s>>>(a.ii, a.jj, (int)W.E, (int)W.K, W.t0, W.t1, a.eta_rows, W.w, a.info);
    HS2_LAUNCH_CHECK("ba_keys_kernel");
  }
  HS2_CUDA(cudaStreamSynchronize(s));
  *grid = pl.hdr.grid;
  return HS2_OK;
}

extern "C" int hs2_ba_batch_run(void* workspace, int num_windows, int grid, int iterations, float lm, float ep,
                                hs2_stream_t stream) {
  using namespace hs2;
  if (!workspace || iterations < 0 || num_windows <= 0 || grid <= 0) {
    set_error("ba_batch_run: null workspace, no windows, no grid or negative iterations");
    return HS2_ERR_INVALID;
  }
  int rc;
  if ((rc = bind_device(workspace))) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  char* base = static_cast<char*>(workspace);
  const int nwin = num_windows;
  size_t o = 0;
  auto take = [&](size_t bytes) { size_t at = o; o = align256(o + bytes); return at; };
  const size_t off_hdr = take(sizeof(BatchHdr));
  const size_t off_wins = take(sizeof(BatchWin) * nwin);
  const size_t off_prefix = take(sizeof(int) * kBatchPhases * (nwin + 1));
  const size_t ctl_bytes = sizeof(unsigned) * (kBatchPhases * (size_t)nwin + 2);
  const size_t off_ctl = take(ctl_bytes);
  const BatchHdr* dh = reinterpret_cast<const BatchHdr*>(base + off_hdr);
  const BatchWin* dw = reinterpret_cast<const BatchWin*>(base + off_wins);
  const int* dp = reinterpret_cast<const int*>(base + off_prefix);
  unsigned* done = reinterpret_cast<unsigned*>(base + off_ctl);
  unsigned* next = done + kBatchPhases * nwin;
  int* abort_flag = reinterpret_cast<int*>(next + 1);
  for (int it = 0; it < iterations; ++it) {
    HS2_CUDA(cudaMemsetAsync(done, 0, ctl_bytes, s));
    void* args[] = {&dh, &dw, &dp, &done, &next, &abort_flag, &lm, &ep};
    HS2_PROF("ba_batch", s);
    HS2_CUDA(cudaLaunchCooperativeKernel((const void*)ba_batch_kernel, dim3(grid), dim3(kBatchThreads), args,
                                         kBatchDynSmem, s));
    HS2_LAUNCH_CHECK("ba_batch_kernel");
    ba_batch_flag_kernel<<<1, 64, 0, s>>>(dw, nwin, abort_flag);
    HS2_LAUNCH_CHECK("ba_batch_flag_kernel");
  }
  return HS2_OK;
}

extern "C" int hs2_ba_batch_set_wait_test(unsigned spin_limit, int unsatisfiable) {
  using namespace hs2;
  const unsigned spin = spin_limit == 0 ? kBatchSpin : spin_limit;
  const unsigned add = unsatisfiable ? 1u : 0u;
  HS2_CUDA(cudaMemcpyToSymbol(g_batch_spin, &spin, sizeof(spin)));
  HS2_CUDA(cudaMemcpyToSymbol(g_batch_unsatisfiable, &add, sizeof(add)));
  return HS2_OK;
}
