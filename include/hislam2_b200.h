/*
 * hislam2_b200 — C ABI of the B200 (sm_100a) dense-BA + correlation operators.
 *
 * Each entry point replaces one operator of HI-SLAM2's compiled extension
 * `droid_backends` (bound in src/droid.cpp:325-341 of the reference).  The
 * signatures take plain device pointers, sizes and a CUDA stream; nothing here
 * depends on PyTorch.  All tensors are dense, row-major ("contiguous") and live
 * on the device that owns them; work is enqueued on `stream` and the calls do
 * not synchronise unless stated.
 *
 * Return value: HS2_OK or an HS2_ERR_* code; hs2_last_error() gives the message
 * (thread-local).  Errors that depend on device-resident data (an edge index out
 * of range, a wrong eta height) are reported in the `info` words, which the
 * kernels write and the caller reads after the stream has drained.
 */
#ifndef HISLAM2_B200_H_
#define HISLAM2_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* hs2_stream_t; /* == cudaStream_t; NULL = legacy default stream */

enum hs2_status {
  HS2_OK = 0,
  HS2_ERR_INVALID = 1,   /* bad sizes / arguments detected on the host */
  HS2_ERR_CUDA = 2,      /* a CUDA runtime call or launch failed */
  HS2_ERR_WORKSPACE = 3, /* workspace pointer missing or too small */
  HS2_ERR_DTYPE = 4      /* unsupported element type */
};

enum hs2_dtype { HS2_F32 = 0, HS2_F16 = 1, HS2_BF16 = 2, HS2_F64 = 3 };

/* Bits of info[0] written on the device. */
enum hs2_device_error {
  HS2_DEV_BAD_INDEX = 1, /* an edge index lies outside the pose/disparity buffers or >= t1 */
  HS2_DEV_BAD_ETA = 2,   /* eta has neither M nor 1 rows (M = #distinct depth frames) */
  HS2_DEV_TIMEOUT = 4,   /* a bounded wait inside a kernel gave up (results are not valid) */
  HS2_DEV_LIMIT = 8,     /* a per-kernel size limit was exceeded (results are not valid) */
  HS2_DEV_NOT_PD = 16    /* a system to be factorised was not positive definite (hs2_jdsa) */
};

/* Message of the last failing call on this thread ("" if none). */
const char* hs2_last_error(void);
/* ABI version, (major << 16) | minor. */
int hs2_version(void);

/* ---------------------------------------------------------------------------
 * frame_distance  (reference: src/droid.cpp:200-216, src/droid_kernels.cu:860-994,2047-2069)
 *   poses [num_poses,7] f32, disps [num_disps,ht,wd] f32, intrinsics [4] f32,
 *   ii/jj [num_edges] int64  ->  dist [num_edges] f32.
 *   info: int32[1] on the device; info[0] |= HS2_DEV_BAD_INDEX for an edge whose
 *   index is outside the buffers (its dist is then 1000).
 */
int hs2_frame_distance(const float* poses, int64_t num_poses, const float* disps, int64_t num_disps,
                       int ht, int wd, const float* intrinsics, const int64_t* ii, const int64_t* jj,
                       int64_t num_edges, float beta, float* dist, int32_t* info, hs2_stream_t stream);

/* ---------------------------------------------------------------------------
 * corr_index_forward  (reference: src/droid.cpp:254-264, src/correlation_kernels.cu:19-70,127-154)
 *   volume [n,h1,w1,h2,w2] of `dtype`, coords [n,2,h1,w1] f32
 *   -> corr [n,2r+1,2r+1,h1,w1] of `dtype` (dim 1 along x, dim 2 along y).
 *   Every element of corr is written (no pre-zeroing needed).
 */
int hs2_corr_index_forward(const void* volume, int dtype, int64_t n, int h1, int w1, int h2, int w2,
                           const float* coords, int radius, void* corr, hs2_stream_t stream);

/* corr_index_backward  (reference: src/droid.cpp:266-275, src/correlation_kernels.cu:73-124,156-184)
 *   coords [n,2,h1,w1] f32, corr_grad [n,2r+1,2r+1,h1,w1] of `dtype`
 *   -> volume_grad [n,h1,w1,h2,w2] of `dtype`, fully written (zeros outside the windows).
 */
int hs2_corr_index_backward(const float* coords, const void* corr_grad, int dtype, int64_t n, int h1,
                            int w1, int h2, int w2, int radius, void* volume_grad, hs2_stream_t stream);

/* ---------------------------------------------------------------------------
 * ba_batch  (callers: hislam2/factor_graph.py:190-235 runs one ba per window;
 * this solves many independent windows at once, each with the semantics of
 * hs2_ba / src/droid_kernels.cu:1820-1937)
 *   One hs2_ba_window per window, with its own device buffers and sizes (any grid,
 *   keyframe and edge count; at most 256 optimised poses).  motion_only is not
 *   supported.  hs2_ba_batch_prepare (synchronous on `stream`, not for capture)
 *   builds the plan and each window's keys in the workspace and returns the grid of
 *   the persistent launch; the window list must not change afterwards.
 *   hs2_ba_batch_run enqueues `iterations` LM iterations, ONE cooperative
 *   persistent kernel launch per iteration over all windows (capturable into a CUDA
 *   graph): poses, disps updated in place, dx / dz written as hs2_ba does.
 *   gram_split: pixel splits per depth frame of the Schur Gram (tuning knob, >= 1);
 *   ctas_per_sm: CTAs per SM of the persistent grid (0 = as many as fit).
 *   Each window's info [4] is as for hs2_ba.
 */
typedef struct hs2_ba_window {
  float* poses;
  int64_t num_poses;
  float* disps;
  int64_t num_disps;
  int ht, wd;
  const float* intrinsics;
  const float* targets;
  const float* weights;
  const float* eta;
  int64_t eta_rows;
  const int64_t* ii;
  const int64_t* jj;
  int64_t num_edges;
  int t0, t1;
  float* dx;
  float* dz;
  int64_t dz_rows;
  int32_t* info;
} hs2_ba_window;
int hs2_ba_batch_workspace_size(const hs2_ba_window* windows, int num_windows, size_t* bytes);
int hs2_ba_batch_prepare(const hs2_ba_window* windows, int num_windows, int gram_split, int ctas_per_sm,
                         void* workspace, size_t workspace_bytes, int* grid, hs2_stream_t stream);
int hs2_ba_batch_run(void* workspace, int num_windows, int grid, int iterations, float lm, float ep,
                     hs2_stream_t stream);
/* Test hook of the batched kernel's bounded waits (current device, synchronous):
 * spin_limit polls before a dependency wait gives up (0 = the default, about a
 * second); unsatisfiable != 0 makes every wait need one completion more than can
 * happen, so that each runs out and the launch reports HS2_DEV_TIMEOUT in every
 * window's info.  Reset with (0, 0). */
int hs2_ba_batch_set_wait_test(unsigned spin_limit, int unsatisfiable);

/* ---------------------------------------------------------------------------
 * ba_adjoint  (no operator of the reference: HI-SLAM2 differentiates its BA only
 * through the pure-PyTorch path, hislam2/geom/ba.py + geom/chol.py:8-22)
 *   Gradients of L(dx, dz) for ONE iteration of hs2_ba (motion_only = 0) with
 *   respect to targets, weights [num_edges,2,ht,wd] and eta [eta_rows,ht,wd], at the
 *   linearisation point poses/disps (those of the step, before it was applied):
 *   implicit differentiation through the damped Schur solve, using the same
 *   system build and Cholesky as the forward.  dx [t1-t0,6] is the step's output,
 *   grad_dx [t1-t0,6] and grad_dz [dz_rows = M, ht*wd] are dL/ddx, dL/ddz; lam
 *   [t1-t0,6] receives the adjoint pose solution.  All outputs are fully written.
 *   info as for hs2_ba, plus HS2_DEV_LIMIT when a depth frame has more than 256
 *   optimised rows or an edge pose more than 8 duplicate rows in one frame.
 *   Workspace: hs2_ba_adjoint_workspace_size() bytes.
 */
int hs2_ba_adjoint_workspace_size(int64_t num_poses, int64_t num_disps, int ht, int wd, int64_t num_edges, int t0,
                                  int t1, size_t* bytes);
int hs2_ba_adjoint(const float* poses, int64_t num_poses, const float* disps, int64_t num_disps, int ht, int wd,
                   const float* intrinsics, const float* targets, const float* weights, const float* eta,
                   int64_t eta_rows, const int64_t* ii, const int64_t* jj, int64_t num_edges, int t0, int t1,
                   float lm, float ep, const float* dx, const float* grad_dx, const float* grad_dz, int64_t dz_rows,
                   float* grad_targets, float* grad_weights, float* grad_eta, float* lam, int32_t* info,
                   void* workspace, size_t workspace_bytes, hs2_stream_t stream);

/* ---------------------------------------------------------------------------
 * corr_volume  (reference: hislam2/modules/corr.py:29-38,63-71 -- CorrBlock's
 * all-pairs volume torch.matmul((f1/4)^T, f2/4) and its avg_pool2d pyramid, built by
 * the caller in PyTorch; this entry point replaces that construction)
 *   fmap1 [k1,channels,ht,wd], fmap2 [k2,channels,ht,wd] of `dtype` (HS2_F16 or
 *   HS2_BF16), ii/jj [num_pairs] int64 (frame of fmap1 / fmap2 of each pair)
 *   -> pyramid[l] [num_pairs, ht, wd, ht>>l, wd>>l] of `dtype` for l < levels (<= 4):
 *   level 0 = sum_c (fmap1[ii,c]/4)(fmap2[jj,c]/4) accumulated in F32 on the tensor
 *   cores, level l = 2x2 average of level l-1 (floor sizes), each level rounded to
 *   `dtype` and pooled from the rounded level above (avg_pool2d's arithmetic).
 *   precision HS2_CV_NATIVE contracts the 16-bit values as given; HS2_CV_E4M3
 *   quantises each pixel's feature vector to FP8 e4m3 with its own scale
 *   (max |f/4| / 448) and rescales the F32 sums.  channels must be 128, wd <= 96.
 *   info: int32[1] on the device; info[0] |= HS2_DEV_BAD_INDEX for a pair whose frame
 *   index is outside [0, k1) / [0, k2) (its outputs are left unwritten),
 *   HS2_DEV_TIMEOUT if a bounded wait gave up.
 *   Workspace: hs2_corr_volume_workspace_size() bytes (the packed operands).
 */
enum hs2_corr_precision { HS2_CV_NATIVE = 0, HS2_CV_E4M3 = 1 };
int hs2_corr_volume_workspace_size(int64_t k1, int64_t k2, int channels, int ht, int wd, int dtype, int precision,
                                   size_t* bytes);
int hs2_corr_volume(const void* fmap1, int64_t k1, const void* fmap2, int64_t k2, int channels, int ht, int wd,
                    int dtype, const int64_t* ii, const int64_t* jj, int64_t num_pairs, int precision, int levels,
                    void* const* pyramid, int32_t* info, void* workspace, size_t workspace_bytes,
                    hs2_stream_t stream);

/* ---------------------------------------------------------------------------
 * corr_reproject_lookup  (reference: the caller side of the update step,
 * hislam2/depth_video.py:170-178 reproject + hislam2/modules/corr.py:90-117
 * AltCorrBlock, as factor_graph.py:194-200,253-260 chain them)
 *   poses [num_poses,7], disps [num_disps,ht,wd], intrinsics [4] f32; fmap_levels[l]
 *   [num_frames,channels,ht>>l,wd>>l] of `dtype` (level 0 = the features, l > 0 their
 *   2x2 average pools); ii/jj [num_edges] int64
 *   -> corr [num_edges, levels*(2r+1)^2, ht, wd] of `dtype`: the pixels of frame ii
 *   projected into frame jj (Gij = Gj Gi^-1), scaled by 2^-l, and the bilinear
 *   radius-r window of (f_ii/4).(f_jj,l/4) at every level -- one launch, no
 *   coordinates or volume in memory.  coords1 [num_edges,ht,wd,2] f32 (optional,
 *   NULL to skip) receives the level-0 coordinates.  info int32[1]:
 *   HS2_DEV_BAD_INDEX for an edge outside the buffers (its outputs are zero).
 */
int hs2_corr_reproject_lookup(const float* poses, int64_t num_poses, const float* disps, int64_t num_disps,
                              const float* intrinsics, const void* const* fmap_levels, int levels, int dtype,
                              int64_t num_frames, int channels, int ht, int wd, const int64_t* ii, const int64_t* jj,
                              int64_t num_edges, int radius, void* corr, float* coords1, int32_t* info,
                              hs2_stream_t stream);

/* The same op on channel-last features (float16 / bfloat16, channels == 128, radius <= 8):
 * packed_levels[l] are hs2_altcorr_pack buffers of the pooled features [1, num_frames,
 * (ht>>l)*(wd>>l), 128] (level 0 must hold the frames of ii and jj, the other levels
 * those of jj).  Each CTA takes an 8x8 block of pixels of one edge and level, reprojects
 * them (the formula above), and computes the block's windows by the staged-box tensor-core
 * product of hs2_altcorr_forward_packed; same outputs. */
int hs2_corr_reproject_lookup_packed(const float* poses, int64_t num_poses, const float* disps, int64_t num_disps,
                                     const float* intrinsics, const void* const* packed_levels, int levels, int dtype,
                                     int64_t num_frames, int channels, int ht, int wd, const int64_t* ii,
                                     const int64_t* jj, int64_t num_edges, int radius, void* corr, float* coords1,
                                     int32_t* info, hs2_stream_t stream);

/* ---------------------------------------------------------------------------
 * altcorr_forward  (reference: src/droid.cpp:277-289, src/altcorr_kernel.cu:25-75,132-172)
 *   fmap1 [b,n1,c,h,w], fmap2 [b,n2,c,h2,w2] of `dtype`, coords [b,m,2,h,w] f32,
 *   ii/jj [m] int64 (frame of fmap1 / fmap2 for each of the m correlations)
 *   -> corr [b,m,2r+1,2r+1,h,w] of `dtype`, dim 2 along x and dim 3 along y,
 *   values (f1/4).(f2/4) bilinearly sampled.  Written densely (contiguous).
 *   info: int32[1]; HS2_DEV_BAD_INDEX for an ii/jj outside [0,n1)/[0,n2) (that
 *   correlation is then all zeros).
 */
int hs2_altcorr_forward(const void* fmap1, const void* fmap2, int dtype, int b, int n1, int n2, int c,
                        int h, int w, int h2, int w2, const float* coords, const int64_t* ii,
                        const int64_t* jj, int m, int radius, void* corr, int32_t* info,
                        hs2_stream_t stream);

/* altcorr_forward on channel-last features (same reference op; float16 / bfloat16 with
 * c in {32, 64, 128, 256}).  hs2_altcorr_pack writes fmap [b,n,c,h,w] channel-last,
 * [b,n,h*w,c], into the start of `workspace` (hs2_altcorr_pack_workspace_size() bytes,
 * a frame-flag array at its end): only the frames listed in `frames[num_frames]` (the
 * ii or jj of a call), or all n frames when `frames` is null.  hs2_altcorr_forward_packed
 * then takes two such buffers in place of fmap1 / fmap2 and writes the same corr as
 * hs2_altcorr_forward: products of the 16-bit features formed exactly and summed in
 * FP32 (the reference rounds each product to the feature type first), window rows read
 * as contiguous channel vectors.  A caller that looks up many edge chunks against one
 * pyramid (AltCorrBlock) packs each level once.
 */
int hs2_altcorr_pack_workspace_size(int dtype, int b, int n, int c, int h, int w, size_t* bytes);
int hs2_altcorr_pack(const void* fmap, int dtype, int b, int n, int c, int h, int w, const int64_t* frames,
                     int num_frames, void* workspace, size_t workspace_bytes, hs2_stream_t stream);
int hs2_altcorr_forward_packed(const void* packed1, const void* packed2, int dtype, int b, int n1, int n2, int c,
                               int h, int w, int h2, int w2, const float* coords, const int64_t* ii,
                               const int64_t* jj, int m, int radius, void* corr, int32_t* info,
                               hs2_stream_t stream);

/* altcorr_backward  (reference: src/droid.cpp:291-305, src/altcorr_kernel.cu:79-129,175-225;
 *   effective positional order as called from hislam2/modules/corr.py:86)
 *   grad [b,m,2r+1,2r+1,h,w] f32 (same layout as the forward output).
 *   -> fmap1_grad [b,n1,c,h,w], fmap2_grad [b,n2,c,h2,w2] of `dtype`, fully written.
 *   `scale` multiplies every product: 1 reproduces the reference operator (which
 *   leaves out the forward's 1/16), 1/16 gives the exact adjoint of the forward.
 *   workspace: f32 accumulators, hs2_altcorr_backward_workspace_size() bytes
 *   (0 when dtype is f32).
 */
int hs2_altcorr_backward_workspace_size(int dtype, int b, int n1, int n2, int c, int h, int w, int h2,
                                        int w2, size_t* bytes);
int hs2_altcorr_backward(const void* fmap1, const void* fmap2, int dtype, int b, int n1, int n2, int c,
                         int h, int w, int h2, int w2, const float* coords, const int64_t* ii,
                         const int64_t* jj, int m, const float* grad, int radius, float scale,
                         void* fmap1_grad, void* fmap2_grad, int32_t* info, void* workspace,
                         size_t workspace_bytes, hs2_stream_t stream);

/* ---------------------------------------------------------------------------
 * ba  (reference: src/droid.cpp:141-168, src/droid_kernels.cu:1820-1937)
 *   Runs `iterations` damped Gauss-Newton steps over the poses [t0,t1) and the
 *   disparity maps of every frame in unique(cat(arange(t0,t1), ii)), updating
 *   `poses` [num_poses,7] and `disps` [num_disps,ht,wd] IN PLACE.
 *   intrinsics [4] f32 (one pinhole camera), targets/weights [num_edges,2,ht,wd] f32,
 *   eta [eta_rows,ht,wd] f32 with eta_rows == M or 1, ii/jj [num_edges] int64,
 *   every ii/jj in [0, min(num_poses,num_disps)) and < t1.
 *   Outputs of the last iteration: dx [t1-t0,6] f32 and, unless motion_only,
 *   dz [M,ht*wd] f32 (dz must hold dz_rows >= M rows; M <= min(num_poses, t1-t0+num_edges)).
 *   info: int32[4] on the device: [0] HS2_DEV_* bits, [1] M, [2] number of
 *   iterations whose Cholesky factorisation failed (their dx is 0, as in the
 *   reference), [3] reserved.  When info[0] != 0 nothing was modified.
 *   workspace: hs2_ba_workspace_size() bytes, 256-byte aligned.
 *   No host synchronisation.
 */
int hs2_ba_workspace_size(int64_t num_poses, int64_t num_disps, int ht, int wd, int64_t num_edges,
                          int t0, int t1, int motion_only, size_t* bytes);
int hs2_ba(float* poses, int64_t num_poses, float* disps, int64_t num_disps, int ht, int wd,
           const float* intrinsics, const float* targets, const float* weights, const float* eta,
           int64_t eta_rows, const int64_t* ii, const int64_t* jj, int64_t num_edges, int t0, int t1,
           int iterations, float lm, float ep, int motion_only, float* dx, float* dz, int64_t dz_rows,
           int32_t* info, void* workspace, size_t workspace_bytes, hs2_stream_t stream);

/* ---------------------------------------------------------------------------
 * pgba  (reference: src/droid.cpp:171-196, src/droid_kernels.cu:1940-2044)
 *   ONE damped Gauss-Newton step over the Sim3 poses [t0,t1) and the disparity maps
 *   of every frame in unique(cat(arange(t0,t1), ii)).  poses [num_poses,8] f32
 *   (t, q xyzw, s) are only read: dx [t1-t0,7] f32 (tangent [tau, phi, sigma]) is
 *   returned for the caller's Sim3 retraction; disps [num_disps,ht,wd] is updated
 *   IN PLACE by dz.  The relative-pose factors: Hsp [4,num_factors,7,7] f32 (blocks
 *   at (iip,iip), (iip,jjp), (jjp,iip), (jjp,jjp)), vsp [2,num_factors,7] f32 (at iip,
 *   jjp), iip/jjp [num_factors] int64 < t1; keys below t0 are dropped as in the
 *   reference.  intrinsics, targets, weights, eta, ii, jj as for hs2_ba.
 *   dz [M,ht*wd] f32 with dz_rows >= min(num_poses, num_disps, t1-t0+num_edges).
 *   info: int32[4] on the device: [0] HS2_DEV_* bits (HS2_DEV_BAD_INDEX also for
 *   iip/jjp >= t1), [1] M, [2] 1 when the factorisation failed (dx = 0, as in the
 *   reference).  When info[0] != 0 disps is unchanged.
 *   workspace: hs2_pgba_workspace_size() bytes, 256-byte aligned.
 */
int hs2_pgba_workspace_size(int64_t num_poses, int64_t num_disps, int ht, int wd, int64_t num_edges,
                            int t0, int t1, size_t* bytes);
int hs2_pgba(const float* poses, int64_t num_poses, float* disps, int64_t num_disps, int ht, int wd,
             const float* intrinsics, const float* targets, const float* weights, const float* eta,
             int64_t eta_rows, const float* Hsp, const float* vsp, const int64_t* iip, const int64_t* jjp,
             int64_t num_factors, const int64_t* ii, const int64_t* jj, int64_t num_edges, int t0, int t1,
             float lm, float ep, float* dx, float* dz, int64_t dz_rows, int32_t* info, void* workspace,
             size_t workspace_bytes, hs2_stream_t stream);

/* ba without allocation.  No counterpart in the reference: this entry point is for
 * callers that cannot allocate device memory when they run a BA step (a process with
 * a GPU memory budget fixed at start-up, a foreign-language host without a caching
 * allocator, for which cudaMalloc / cudaFree in the tracking loop would stall the
 * device).  Same arguments
 * and results as hs2_ba, minus the workspace: the scratch is a static device array
 * of 64 MiB inside the library, held by every GPU that loads it until exit.
 * Problems whose hs2_ba_workspace_size() exceeds 64 MiB are rejected with
 * HS2_ERR_WORKSPACE.  The first call on a device looks up the array's address
 * (make that call before any stream capture).  All calls share the array, so calls
 * whose GPU work overlaps in time race and must be serialised by the caller.
 */
int hs2_ba_noalloc(float* poses, int64_t num_poses, float* disps, int64_t num_disps, int ht, int wd,
                   const float* intrinsics, const float* targets, const float* weights, const float* eta,
                   int64_t eta_rows, const int64_t* ii, const int64_t* jj, int64_t num_edges, int t0,
                   int t1, int iterations, float lm, float ep, int motion_only, float* dx, float* dz,
                   int64_t dz_rows, int32_t* info, hs2_stream_t stream);

/* Key generation of ba alone, for parity checks of the integer keys
 * (reference: src/droid_kernels.cu:1841-1849 unique/inverse, :1712-1740 schur rows).
 *   kx [min(num_poses,t1-t0+num_edges)] int32: sorted distinct frames of cat(arange(t0,t1), ii);
 *   kk_exp [t1-t0+num_edges] int32: inverse index of each row of cat(arange(t0,t1), ii);
 *   rows_ptr [num_rows_cap+1] / rows [t1-t0+num_edges] int32: per depth slot k, the rows
 *   n (0..t1-t0+num_edges) whose pose jj_exp[n] lies in [t0,t1), in increasing n.
 *   info as for hs2_ba.  Uses the same workspace as hs2_ba.
 */
int hs2_ba_keys(int64_t num_poses, int64_t num_disps, int ht, int wd, const int64_t* ii,
                const int64_t* jj, int64_t num_edges, int t0, int t1, int32_t* kx, int32_t* kk_exp,
                int32_t* rows_ptr, int32_t* rows, int32_t* info, void* workspace,
                size_t workspace_bytes, hs2_stream_t stream);

/* The reduced camera system of one linearisation, for block-level parity checks
 * (reference: the matrix (A - S) and vector (A.b - S.b) handed to
 * SparseBlock::solve at src/droid_kernels.cu:1909, before damping).
 *   A_out [6(t1-t0), 6(t1-t0)] f64 row-major (full symmetric), b_out [6(t1-t0)] f64;
 *   motion_only gives the pose block A alone (src/droid_kernels.cu:1878-1898).
 *   Arguments otherwise as for hs2_ba; poses and disps are not modified.
 */
int hs2_ba_reduced_system(const float* poses, int64_t num_poses, const float* disps, int64_t num_disps,
                          int ht, int wd, const float* intrinsics, const float* targets,
                          const float* weights, const float* eta, int64_t eta_rows, const int64_t* ii,
                          const int64_t* jj, int64_t num_edges, int t0, int t1, int motion_only,
                          double* A_out, double* b_out, int32_t* info, void* workspace,
                          size_t workspace_bytes, hs2_stream_t stream);

/* ---------------------------------------------------------------------------
 * iproj  (reference: src/droid.cpp:233-242, src/droid_kernels.cu:1208-1272,2120-2143)
 * points[b,i,j,:] = (R_b X + d t_b) / d with X = ((j-cx)/fx, (i-cy)/fy, 1), d = disps[b,i,j],
 * for every frame b of disps (poses must have at least num_disps rows).  points: [N,H,W,3] f32.
 */
int hs2_iproj(const float* poses, int64_t num_poses, const float* disps, int64_t num_disps, int ht, int wd,
              const float* intrinsics, float* points, hs2_stream_t stream);

/* covis_distance  (reference: src/droid.cpp:218-231, src/droid_kernels.cu:996-1090,2071-2091)
 * dist[n] = fraction of frame i = ii[n]'s pixels that project outside the image under both
 * Gj Gi^-1 with j = i-1 and j = i+1.  Entries with i < 1 or i+1 >= num_poses or
 * i >= num_disps set HS2_DEV_BAD_INDEX in info[0] (the reference reads out of bounds).
 */
int hs2_covis_distance(const float* poses, int64_t num_poses, const float* disps, int64_t num_disps, int ht,
                       int wd, const float* intrinsics, const int64_t* ii, int64_t num, float* dist, int32_t* info,
                       hs2_stream_t stream);

/* depth_filter  (reference: src/droid.cpp:308-322, src/droid_kernels.cu:1094-1204,2093-2118)
 * counter[b,i,j] (zeroed here) = number of neighbours k in {i-1,i-2,i-3,i+3,i+4,i+5} of frame
 * i = ix[b] (inside the buffer) in which pixel (i,j)'s reprojected inverse depth lies within
 * thresh[b] of one of the four disparities around the reprojection.  Needs num_poses >=
 * num_disps; ix outside [0, num_disps) sets HS2_DEV_BAD_INDEX.
 */
int hs2_depth_filter(const float* poses, int64_t num_poses, const float* disps, int64_t num_disps, int ht, int wd,
                     const float* intrinsics, const int64_t* ix, const float* thresh, int64_t num, float* counter,
                     int32_t* info, hs2_stream_t stream);

/* proj_trans  (reference: src/droid.cpp:121-139, src/droid_kernels.cu:246-362,1781-1818)
 * Depth-only Schur terms of the mono-prior alignment: per edge e and pixel,
 * C = wu Jzu^2 + wv Jzv^2 and w = wu ru Jzu + wv rv Jzv (the ba linearisation without the
 * pose blocks), summed into row slot[e] of C, w [num_slots, H*W] (zeroed here).  The
 * reference sums over kx = unique(ii) (accum_cuda); slot[e] is the position of ii[e] in kx.
 * intrinsics: the 4 values of the camera (the reference reads row 0 of an [N,4] tensor).
 */
int hs2_proj_trans(const float* poses, int64_t num_poses, const float* disps, int64_t num_disps, int ht, int wd,
                   const float* intrinsics, const float* targets, const float* weights, const int64_t* ii,
                   const int64_t* jj, const int64_t* slot, int64_t num_edges, int64_t num_slots, float* C, float* w,
                   int32_t* info, hs2_stream_t stream);

/* bi_inter  (reference: src/droid.cpp:244-251, src/droid_kernels.cu:1275-1316,2145-2175)
 * outputs[b,i,j] = bilinear interpolation of scales[b] ([hs, ws]) at grids[b,i,j] = (x, y),
 * jacobians[b,i,j] ([hs, ws], zeroed here) = its four interpolation weights.  Grid points
 * whose 2x2 cell leaves the scale grid set HS2_DEV_BAD_INDEX (the reference writes out of
 * bounds there).
 */
int hs2_bi_inter(const float* scales, int64_t num, int hs, int ws, const float* grids, int ht, int wd,
                 float* outputs, float* jacobians, int32_t* info, hs2_stream_t stream);

/* jdsa  (reference: hislam2/geom/ba.py:170-219 JDSA, :159-167 get_prior_depth_aligned,
 *        hislam2/geom/chol.py:80-107 schur_solve_mono_prior; the caller is
 *        hislam2/depth_video.py:234-240)
 * One mono-prior depth / scale alignment step after ba: proj_trans's C, w of the edges
 * (ii, jj), the prior terms of disps_prior [num_prior, H, W] aligned by the per-frame
 * bilinear scale grids dscales [num_scales, hs, ws], a damped solve (ep 0.1, lm 1e-4) for
 * the hs*ws scale unknowns of every source frame and the depth update by back-substitution.
 *   disps [num_disps, H, W] is read only; disps_out [num_disps, H, W] receives
 *   clamp(where(d > 10, 0, d), min = 0.001) of every frame, d = disps + dz on the source
 *   frames.  dscales[kx[b]] += dso[b] in place.  dso [M, hs*ws] and dzcov [M, H*W] (may be
 *   NULL) are outputs; C, w [M, H*W] are scratch.  M = num_kx.
 *   kx [M]: the sorted distinct values of ii; slot [num_edges]: the position of ii[e] in kx
 *   (torch.unique(ii, return_inverse=True)).  eta: M*H*W values (row b for frame kx[b]).
 *   grid_y [ht] = linspace(0, hs-1-1e-6, ht), grid_x [wd] = linspace(0, ws-1-1e-6, wd), in
 *   float32 as torch.linspace computes them (the reference's sampling grid).
 *   Limits: 2 <= hs, ws; hs*ws <= 16; ht, wd <= 4096; 1 <= M <= 65535.
 *   info: int32[1], zeroed here; HS2_DEV_BAD_INDEX for an edge or kx outside the buffers, an
 *   unsorted kx or a grid point whose 2x2 cell leaves the scale grid; HS2_DEV_NOT_PD when a
 *   block of the reduced system is not positive definite (the reference raises there, in
 *   torch.linalg.inv of the zero factor its CholeskySolver returns).  With either bit set
 *   dscales is left unchanged and disps_out is not valid.
 */
int hs2_jdsa(const float* poses, int64_t num_poses, const float* disps, int64_t num_disps, int ht, int wd,
             const float* intrinsics, const float* targets, const float* weights, const float* eta,
             const float* disps_prior, int64_t num_prior, float* dscales, int64_t num_scales, int hs, int ws,
             const float* grid_y, const float* grid_x, const int64_t* ii, const int64_t* jj, const int64_t* slot,
             int64_t num_edges, const int64_t* kx, int64_t num_kx, float alpha, float* C, float* w, float* dso,
             float* disps_out, float* dzcov, int32_t* info, hs2_stream_t stream);

/* pgo_constraints  (reference: hislam2/pgo_buffer.py:39-63 global_relative_posesim3_constraints,
 *                   called at hislam2/depth_video.py:259 before every pgba step)
 * Blocks of the relative Sim3 pose factors for hs2_pgba: per factor n, the residual
 * r = log(Gij Gi Gj^-1) with Gi = poses[ii[n]], Gj = poses[jj[n]] (Sim3 [t, q xyzw, s]) and
 * Gij = rel_poses[n] (SE3 [t, q], scale 1), its Jacobians w.r.t. exp(d) Gi and exp(d) Gj
 * by central differences of step 1e-8 in FP64 (the reference's numeric Jacobians), then
 * wJx^T = float((pw Jx)^T info) and
 *   Hsp [4, num_factors, 7, 7] = [wJi^T Ji, wJi^T Jj, wJj^T Ji, wJj^T Jj],
 *   vsp [2, num_factors, 7] = -[wJi^T r, wJj^T r],  chi [num_factors, 2] = (r.r, r.info r)
 * in float32 (sum chi over the factors for the reference's chi2 / chi2_scaled).
 *   infos [num_factors, 7, 7] f32.  info: int32[1], zeroed here; HS2_DEV_BAD_INDEX for a
 *   factor whose ii / jj is outside [0, num_poses) (its blocks are zero).
 */
int hs2_pgo_constraints(const float* poses, int64_t num_poses, const int64_t* ii, const int64_t* jj,
                        const float* rel_poses, const float* infos, int64_t num_factors, double pw, float* Hsp,
                        float* vsp, float* chi, int32_t* info, hs2_stream_t stream);

/* sim3_retr  (reference: hislam2/geom/ba.py:27-29 pose_retr on Sim3 poses, lietorch's retr;
 *             called at hislam2/depth_video.py:267 after every pgba step)
 * poses[t0 + k] <- exp(dx[k]) poses[t0 + k] for k < t1 - t0, in place; poses [num_poses, 8]
 * Sim3 f32, dx [t1 - t0, 7] f32 (pgba's dx).  Computed in FP64, stored as float.
 */
int hs2_sim3_retr(float* poses, int64_t num_poses, const float* dx, int64_t t0, int64_t t1, hs2_stream_t stream);

/* Selects the kernels of the linearisation and Schur Gram for later hs2_ba calls
 * (process-wide; no counterpart in the reference, whose Gram is SIMT FP32 in
 * EEt6x6_kernel):
 *   0 (default) linearisation writing the E rows, then their Gram on tensor cores
 *     (tcgen05 kind::tf32 with a hi/lo split of both operands: 3 products, about FP32
 *     accuracy); frames with more than 42 Schur rows use the SIMT Gram.  Needs
 *     eta > 0 (Q = 1/(C+eta) >= 0);
 *   1 SIMT FP32 Gram for every frame;
 *   2 one fused kernel per depth frame: linearisation and the tensor-core Gram of its
 *     E rows straight from shared memory; the back-substitution recomputes E.  Frames
 *     with more than 40 edges or 42 Schur rows use the unfused kernels.  Needs eta > 0.
 */
int hs2_ba_set_schur_path(int path);

/* Precision of ba's tensor-core Schur Gram (process-wide, default 1; no counterpart
 * in the reference, whose Gram is FP32 SIMT):
 *   1 3xTF32 (hi.hi + hi.lo + lo.hi): FP32-accurate Hessian blocks;
 *   0 one TF32 product per term: the reduced camera system carries about 1e-3 relative
 *     error while the gradient stays FP32, so Gauss-Newton converges to the same
 *     point (the mixed-precision form; bench.py reports its pose error).
 * Applies to the default Schur path (0 of hs2_ba_set_schur_path); frames on the SIMT
 * Gram (more than 42 Schur rows) and the fused per-frame path keep FP32 accuracy. */
int hs2_ba_set_gram_precision(int precision);

/* ---------------------------------------------------------------------------
 * Measurement support (no counterpart in the reference, which has no profiler).
 * hs2_profile_enable(1) brackets every kernel launch of this library with CUDA
 * events on its stream; hs2_profile_report() waits for them and writes one line
 * per kernel, "<name> <launches> <total_ms>", into buf (returns the text length;
 * reset != 0 clears the record).
 */
void hs2_profile_enable(int on);
/* Number of kernels this library has launched in this process. */
long long hs2_launch_count(void);
int hs2_profile_report(char* buf, size_t len, int reset);

#ifdef __cplusplus
}
#endif

#endif /* HISLAM2_B200_H_ */
